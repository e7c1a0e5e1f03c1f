"""janc_b200: JANC's per-step reacting-flow path (WENO5-JS or MUSCL with LF or
Steger-Warming splitting or a Godunov Riemann solver, viscous and LES fluxes,
SSP-RK3, NASA7 thermo with the Halley temperature solve, point-implicit H2-air
chemistry) as hand-written sm_100a CUDA kernels behind a C ABI
(``include/janc_b200.h``), with Python entry points that keep the reference's
call signatures: ``janc_b200.Solver``, the ``janc_b200.janc`` module mirror,
``janc_b200.slab`` (x slabs over ranks), ``janc_b200.ensemble`` and
``janc_b200.adjoint``.
"""
from . import mechanism  # noqa: F401
from ._native import JancError, lib  # noqa: F401

__version__ = "0.1.0"


def __getattr__(name):
    # torch-dependent modules load lazily so that the mechanism tables and
    # the library loader import without a GPU
    if name == "Solver":
        from .solver import Solver
        return Solver
    raise AttributeError(name)
