"""Time steppers (src/janc_v2/simulation/time_step): SSP-RK3
(TVD_RK3.py:5-12) and Heun's RK2 (RK2.py:5-12).

With the rhs/update functions returned by ``set_rhs`` the whole step runs as
one fused native call (``jb_rk3``); with other callables the three stages are
composed here exactly as the reference writes them."""
from .. import _state


def _tvd_rk3(U, aux, dx, dy, dt, theta, rhs_func, update_func):
    native = getattr(rhs_func, "_janc_b200_flux", False) and getattr(update_func, "_janc_b200_update", False)
    if native:
        Ud, kind = _state.to_device(U)
        auxd, _ = _state.to_device(aux)
        s = _state.solver_for(tuple(Ud.shape[1:]), dx, dy if Ud.ndim == 3 else None)
        U3, aux3 = s.rk3(Ud, auxd, dx, dy if Ud.ndim == 3 else None, float(dt), theta)
        return _state.back(U3, kind), _state.back(aux3, kind)
    U1 = U + rhs_func(U, aux, dx, dy, dt, theta)
    aux1 = update_func(U1, aux)
    U2 = 3 / 4 * U + 1 / 4 * (U1 + rhs_func(U1, aux1, dx, dy, dt, theta))
    aux2 = update_func(U2, aux1)
    U3 = 1 / 3 * U + 2 / 3 * (U2 + rhs_func(U2, aux2, dx, dy, dt, theta))
    aux3 = update_func(U3, aux2)
    return U3, aux3


def _rk2(U, aux, dx, dy, dt, theta, rhs_func, update_func):
    """RK2.py:5-12 (Heun): two rhs evaluations composed as the reference
    writes them, each through the native flux_func / update_aux when those
    are the functions given."""
    dev = rhs_func(U, aux, dx, dy, dt, theta)
    U1 = U + dev
    aux1 = update_func(U1, aux)
    dev1 = rhs_func(U1, aux1, dx, dy, dt, theta)
    U2 = U + 1 / 2 * (dev + dev1)
    aux2 = update_func(U2, aux1)
    return U2, aux2


time_step_dict = {"TVD_RK3": _tvd_rk3, "RK2": _rk2}
