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


_user_source = None


def set_source_terms(user_set):
    """aux_func.py:6-18: the user's source function, or zeros."""
    global _user_source
    fn = None if user_set is None else user_set.get("self_defined_source_terms")
    _user_source = fn


def source_terms(U, aux, theta=None):
    """aux_func.py source_terms: the user's source, zeros without one."""
    if _user_source is None:
        return U * 0
    return _user_source(U, aux, theta)


def aux_to_thermo(U, aux):
    """aux_func.py aux_to_thermo: (gamma, T)."""
    return aux[0:1], aux[1:2]
