"""Time steppers (src/janc_v2/simulation/time_step): SSP-RK3
(TVD_RK3.py:5-12) and Heun's RK2 (RK2.py:5-12), and their block-AMR forms
(TVD_RK3.py:15-36, RK2.py:14-32).

With the rhs/update functions returned by ``set_rhs`` the whole step runs as
one fused native call (``jb_rk3``; for blocks one ``jb_amr_stage`` per
stage); with other callables the stages are composed here exactly as the
reference writes them.

The AMR forms take their blocks' ghost layers from a block layer: the
external ``jaxamr`` package's ``amr.get_ghost_block_data(ref_blk_data,
ref_blk_info)`` and ``amr.update_external_boundary(level, blk_data,
interior, ref_blk_info)`` in the reference.  jaxamr is not part of JANC and
works on JAX arrays; give a layer with those two functions on torch CUDA
tensors to ``set_amr_module`` (or install one importable as
``jaxamr.amr``)."""
from .. import _state

_AMR = {"module": None}


def set_amr_module(module):
    """Use ``module`` (anything with ``get_ghost_block_data`` and
    ``update_external_boundary``) as the block layer of the AMR steps;
    ``None`` returns to importing ``jaxamr.amr``."""
    _AMR["module"] = module


def _amr():
    if _AMR["module"] is not None:
        return _AMR["module"]
    try:
        from jaxamr import amr
    except ImportError as e:
        raise ImportError("the AMR time steps need a block layer (jaxamr's amr.get_ghost_block_data and "
                          "amr.update_external_boundary); none is importable - give one with "
                          "janc.simulation.time_step.set_amr_module") from e
    return amr


def _cat(parts, axis):
    if type(parts[0]).__module__.startswith("torch"):
        import torch
        return torch.cat(parts, dim=axis)
    import numpy as np
    return np.concatenate(parts, axis=axis)


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


def _native_amr(rhs_func, update_func):
    return getattr(rhs_func, "_janc_b200_amr_flux", False) and getattr(update_func, "_janc_b200_amr_update", False)


def _tvd_rk3_amr(level, blk_data, dx, dy, dt, ref_blk_data, ref_blk_info, theta, rhs_func, update_func):
    """TVD_RK3.advance_one_step_amr (TVD_RK3.py:15-36): each stage on the
    blocks with their ghost layers from the block layer, the new interiors
    handed back through update_external_boundary.  With the block functions
    of ``set_rhs(is_amr=True)`` each stage is one native launch
    (``jb_amr_stage``: flux, RK combination and the blocks' temperature
    solves)."""
    amr = _amr()
    if _native_amr(rhs_func, update_func):
        s = _state.solver_for_amr()

        def ghosts(b):
            return _state.to_device(amr.get_ghost_block_data(b, ref_blk_info))[0]
        G0 = ghosts(ref_blk_data)
        B = s.amr_stage(G0, None, 1, dx, dy, dt)
        G1 = ghosts(amr.update_external_boundary(level, blk_data, B[..., 3:-3, 3:-3], ref_blk_info))
        B = s.amr_stage(G1, G0, 2, dx, dy, dt)
        G2 = ghosts(amr.update_external_boundary(level, blk_data, B[..., 3:-3, 3:-3], ref_blk_info))
        B = s.amr_stage(G2, G0, 3, dx, dy, dt)
        return amr.update_external_boundary(level, blk_data, B[..., 3:-3, 3:-3], ref_blk_info)
    g = amr.get_ghost_block_data(ref_blk_data, ref_blk_info)
    U, aux = g[:, 0:-2], g[:, -2:]
    U1 = U + rhs_func(U, aux, dx, dy, dt, theta)
    aux1 = update_func(U1, aux)
    blk1 = amr.update_external_boundary(level, blk_data, _cat([U1, aux1], 1)[..., 3:-3, 3:-3], ref_blk_info)
    g1 = amr.get_ghost_block_data(blk1, ref_blk_info)
    U1, aux1 = g1[:, 0:-2], g1[:, -2:]
    U2 = 3 / 4 * U + 1 / 4 * (U1 + rhs_func(U1, aux1, dx, dy, dt, theta))
    aux2 = update_func(U2, aux1)
    blk2 = amr.update_external_boundary(level, blk_data, _cat([U2, aux2], 1)[..., 3:-3, 3:-3], ref_blk_info)
    g2 = amr.get_ghost_block_data(blk2, ref_blk_info)
    U2, aux2 = g2[:, 0:-2], g2[:, -2:]
    U3 = 1 / 3 * U + 2 / 3 * (U2 + rhs_func(U2, aux2, dx, dy, dt, theta))
    aux3 = update_func(U3, aux2)
    return amr.update_external_boundary(level, blk_data, _cat([U3, aux3], 1)[..., 3:-3, 3:-3], ref_blk_info)


def _rk2_amr(level, blk_data, dx, dy, dt, ref_blk_data, ref_blk_info, theta, rhs_func, update_func):
    """RK2.advance_one_step_amr (RK2.py:14-32), composed as the reference
    writes it (each rhs / update a native call with the block functions of
    ``set_rhs(is_amr=True)``)."""
    amr = _amr()
    g = amr.get_ghost_block_data(ref_blk_data, ref_blk_info)
    U, aux = g[:, 0:-2], g[:, -2:]
    dev = rhs_func(U, aux, dx, dy, dt, theta)
    U1 = U + dev
    aux1 = update_func(U1, aux)
    blk1 = amr.update_external_boundary(level, blk_data, _cat([U1, aux1], 1)[..., 3:-3, 3:-3], ref_blk_info)
    g1 = amr.get_ghost_block_data(blk1, ref_blk_info)
    U1, aux1 = g1[:, 0:-2], g1[:, -2:]
    dev1 = rhs_func(U1, aux1, dx, dy, dt, theta)
    U2 = U + 1 / 2 * (dev + dev1)
    aux2 = update_func(U2, aux1)
    return amr.update_external_boundary(level, blk_data, _cat([U2, aux2], 1)[..., 3:-3, 3:-3], ref_blk_info)


time_step_dict = {"TVD_RK3": _tvd_rk3, "RK2": _rk2, "TVD_RK3_amr": _tvd_rk3_amr, "RK2_amr": _rk2_amr}
