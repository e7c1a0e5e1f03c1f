"""Boundary selection (src/janc_v2/boundary/boundary.py set_boundary).

Named conditions run inside the kernels: periodic, slip_wall, zero_gradient,
no_slip_wall, pressure_outlet, and 'rdc_injector' (the injector of the
reference's example 2, bottom side).  A function on any side is called
before each flux evaluation with the 3 boundary-adjacent layers and theta
and returns the 3 ghost layers (boundary.py:16-21, 37-42, 58-63, 79-84)."""
from .. import _state

_KINDS = ("periodic", "slip_wall", "zero_gradient", "no_slip_wall", "pressure_outlet", "rdc_injector")


def set_boundary(boundary_config, dim):
    keys = ("left_boundary", "right_boundary") + (("bottom_boundary", "top_boundary") if dim == "2D" else ())
    bc = {}
    for k in keys:
        v = boundary_config[k]
        if callable(v):
            bc[k] = v
            continue
        if v not in _KINDS:
            raise KeyError(v)
        bc[k] = v
    _state.config["boundary"] = bc
    _state.config["dim"] = dim


def _padded(U, aux, theta):
    Ud, kind = _state.to_device(U)
    ad, _ = _state.to_device(aux)
    s = _state.solver_for(tuple(Ud.shape[1:]))
    Up, Ap = s.boundary_conditions(Ud, ad, theta)
    return _state.back(Up, kind), _state.back(Ap, kind)


def boundary_conditions_1D(U, aux, theta=None):
    """boundary.py:120-124: the ghost-padded (U, aux), (nv, nx+6), (2, nx+6)."""
    return _padded(U, aux, theta)


def boundary_conditions_2D(U, aux, theta=None):
    """boundary.py:126-132: the ghost-padded (U, aux), (nv, nx+6, ny+6),
    (2, nx+6, ny+6), corners included."""
    return _padded(U, aux, theta)
