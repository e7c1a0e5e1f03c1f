"""Boundary selection (src/janc_v2/boundary/boundary.py set_boundary).

Named conditions run inside the kernels: periodic, slip_wall, zero_gradient,
no_slip_wall, pressure_outlet, and 'rdc_injector' (the injector of the
reference's example 2, bottom side).  A function on the left or right side
is called before each flux evaluation with the 3 boundary-adjacent columns
and theta and returns the 3 ghost columns (boundary.py:16-21, 37-42); on
the bottom or top side it raises NotImplementedError."""
from .. import _state

_KINDS = ("periodic", "slip_wall", "zero_gradient", "no_slip_wall", "pressure_outlet", "rdc_injector")


def set_boundary(boundary_config, dim):
    keys = ("left_boundary", "right_boundary") + (("bottom_boundary", "top_boundary") if dim == "2D" else ())
    bc = {}
    for k in keys:
        v = boundary_config[k]
        if callable(v):
            if k in ("bottom_boundary", "top_boundary"):
                raise NotImplementedError(f"{k}: boundary functions are taken on the left and right sides; "
                                          f"use one of {', '.join(_KINDS)}")
            bc[k] = v
            continue
        if v not in _KINDS:
            raise KeyError(v)
        bc[k] = v
    _state.config["boundary"] = bc
    _state.config["dim"] = dim
