"""Conserved <-> primitive (src/janc_v2/solver_1D/aux_func.py)."""
from .. import _state


def update_aux(U, aux):
    """aux_func.py update_aux: (gamma, T) from the Halley solve."""
    Ud, kind = _state.to_device(U)
    auxd, _ = _state.to_device(aux)
    s = _state.solver_for(tuple(Ud.shape[1:]))
    return _state.back(s.update_aux(Ud, auxd), kind)


def U_to_prim(U, aux):
    """aux_func.py U_to_prim: (rho, u, [v,] Y, p, a)."""
    Ud, kind = _state.to_device(U)
    auxd, _ = _state.to_device(aux)
    s = _state.solver_for(tuple(Ud.shape[1:]))
    return tuple(_state.back(o, kind) for o in s.u_to_prim(Ud, auxd))
