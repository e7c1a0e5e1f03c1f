"""Module state shared by the mirror modules (the reference keeps the same
configuration in module globals), and the cache of native solvers."""
import numpy as np

from .. import mechanism as _mech

config = {
    "mechanism": _mech.DEFAULT_MECHANISM,
    "nondim": None,
    "dim": "2D",
    "boundary": None,
    "precision": "fp64",
    "flux": {"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS",
             "split_method": "LF", "viscosity": "off"},
    "detailed_chemistry": True,
    "transport": None,
    "slab": None,  # janc_b200.slab.Slab of this rank in the is_parallel mode
}
_solvers = {}
_mech_cache = {}


def mechanism():
    key = (config["mechanism"], repr(config["nondim"]))
    if key not in _mech_cache:
        _mech_cache[key] = _mech.load(config["mechanism"], config["nondim"])
    return _mech_cache[key]


def solver_for(shape, dx=1.0, dy=1.0):
    """Cached native solver for a grid shape (1D: (nx,), 2D: (nx, ny))."""
    from ..solver import Solver
    dim = 1 if len(shape) == 1 else 2
    bc = config["boundary"] or {}
    slab = config["slab"]
    key = (dim, tuple(shape), repr(sorted(bc.items())) if bc else "", config["precision"],
           config["mechanism"], repr(config["nondim"]), repr(config["flux"]), repr(config["transport"]),
           None if slab is None else (slab.rank, slab.size, id(slab.group)))
    s = _solvers.get(key)
    if s is None:
        s = Solver(dim, shape[0], shape[1] if dim == 2 else None, dx, dy if dim == 2 else None,
                   bc, mechanism(), precision=config["precision"], flux_config=config["flux"],
                   transport_config=config["transport"], slab=slab)
        _solvers[key] = s
    s._spacing(dx, dy if dim == 2 else None)
    return s


class _Padded:
    """The ghost layers of the padded arrays a padded-input flux call was
    given, served to the solver as its boundary functions."""
    Up = None
    Ap = None

    @staticmethod
    def side(k):
        def fn(U, aux, theta=None):
            Up, Ap = _Padded.Up, _Padded.Ap
            one_d = Up.ndim == 2
            sl = {"left_boundary": (slice(0, 3),) if one_d else (slice(0, 3), slice(3, -3)),
                  "right_boundary": (slice(-3, None),) if one_d else (slice(-3, None), slice(3, -3)),
                  "bottom_boundary": (slice(3, -3), slice(0, 3)),
                  "top_boundary": (slice(3, -3), slice(-3, None))}[k]
            return Up[(slice(None),) + sl], Ap[(slice(None),) + sl]
        return fn


_PADDED_FNS = {k: _Padded.side(k) for k in ("left_boundary", "right_boundary", "bottom_boundary", "top_boundary")}


def solver_for_padded(Up, Ap, dx=1.0, dy=1.0):
    """Cached native solver that takes its ghost layers from the padded
    arrays (Up, Ap) of a total_flux call; returns the solver and the
    contiguous interior (U, aux)."""
    from ..solver import Solver
    dim = Up.ndim - 1
    shape = tuple(n - 6 for n in Up.shape[1:])
    key = ("padded", dim, shape, config["precision"], config["mechanism"], repr(config["nondim"]),
           repr(config["flux"]), repr(config["transport"]))
    s = _solvers.get(key)
    if s is None:
        keys = ("left_boundary", "right_boundary", "bottom_boundary", "top_boundary")[: 2 * dim]
        s = Solver(dim, shape[0], shape[1] if dim == 2 else None, dx, dy if dim == 2 else None,
                   {k: _PADDED_FNS[k] for k in keys}, mechanism(), precision=config["precision"],
                   flux_config=config["flux"], transport_config=config["transport"])
        _solvers[key] = s
    s._spacing(dx, dy if dim == 2 else None)
    _Padded.Up, _Padded.Ap = Up, Ap
    inner = (slice(None), slice(3, -3)) + ((slice(3, -3),) if dim == 2 else ())
    return s, Up[inner].contiguous(), Ap[inner].contiguous()


def solver_for_amr():
    """Cached 2D native solver whose mechanism, precision and flux options
    the block-AMR calls use (its own grid is not used by them)."""
    from ..solver import Solver
    key = ("amr", config["precision"], config["mechanism"], repr(config["nondim"]), repr(config["flux"]),
           repr(config["transport"]))
    s = _solvers.get(key)
    if s is None:
        bc = {k: "periodic" for k in ("left_boundary", "right_boundary", "bottom_boundary", "top_boundary")}
        s = Solver(2, 8, 8, 1.0, 1.0, bc, mechanism(), precision=config["precision"], flux_config=config["flux"],
                   transport_config=config["transport"])
        _solvers[key] = s
    return s


def reset_solvers():
    for s in _solvers.values():
        s.close()
    _solvers.clear()


def to_device(x):
    """(tensor, kind): CUDA float64 contiguous tensor and how to return results."""
    import torch
    if isinstance(x, torch.Tensor):
        return x.to(device="cuda", dtype=torch.float64).contiguous(), "torch"
    if hasattr(x, "__dlpack__") and not isinstance(x, np.ndarray):
        return torch.from_dlpack(x).to(device="cuda", dtype=torch.float64).contiguous(), "torch"
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device="cuda"), "numpy"


def back(t, kind):
    if kind == "numpy":
        return t.detach().cpu().numpy()
    return t
