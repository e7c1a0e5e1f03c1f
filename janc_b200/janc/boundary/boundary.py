"""Boundary selection (src/janc_v2/boundary/boundary.py set_boundary).

Named conditions run inside the kernels: periodic, slip_wall, zero_gradient,
no_slip_wall, pressure_outlet, and 'rdc_injector' (the injector of the
reference's example 2, bottom side).  Python callables cannot run on the GPU
and raise NotImplementedError."""
from .. import _state

_KINDS = ("periodic", "slip_wall", "zero_gradient", "no_slip_wall", "pressure_outlet", "rdc_injector")


def set_boundary(boundary_config, dim):
    keys = ("left_boundary", "right_boundary") + (("bottom_boundary", "top_boundary") if dim == "2D" else ())
    bc = {}
    for k in keys:
        v = boundary_config[k]
        if callable(v):
            raise NotImplementedError(f"{k}: Python callables cannot run inside the kernels; "
                                      f"use one of {', '.join(_KINDS)}")
        if v not in _KINDS:
            raise KeyError(v)
        bc[k] = v
    _state.config["boundary"] = bc
    _state.config["dim"] = dim
