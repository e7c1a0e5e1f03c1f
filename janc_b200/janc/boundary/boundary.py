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
