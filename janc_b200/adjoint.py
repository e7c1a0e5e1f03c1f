"""Reverse mode of the reacting step (2D and 1D) behind ``torch.autograd``.

The reference obtains gradients with ``jax.grad`` through its step
(src/janc_v2/simulation/set_simulator.py:117-122), its CFL time step
(:420-447) and get_T's custom VJP (model/thermo_model.py:155-190).  Here the
forward is the native float64 path and the backward runs hand-written
adjoint kernels (``jb_adjoint_step``) one step at a time in reverse,
recomputing each segment of ``checkpoint`` steps from its stored starting
state (the only states kept by the forward pass).

    traj = Trajectory(solver, cfl=0.05, probe=(x0, y0, 4, 4), checkpoint=20)
    T = T0.clone().requires_grad_()
    lnA = torch.zeros(19, dtype=torch.float64, device="cuda", requires_grad=True)
    dts, pps = probe_trajectory(traj, P, T, Y, lnA, nsteps=200)
    loss = (dts * pps).sum()        # time-integrated probe pressure
    loss.backward()                 # T.grad, lnA.grad

A 1D solver takes the probe as (x0, wx) (cells x0 .. x0 + wx - 1).
"""
import ctypes

import torch

from . import _native
from .solver import Solver, _ptr, _stream

SLOT_DOUBLES = 13  # sizeof(jb_slots) / 8


def _off(t, n):
    """Device pointer to element n of a float64 tensor (None for None)."""
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr() + 8 * n)


class Trajectory:
    """A configured float64 solver (2D or 1D) plus the loss probe and
    checkpointing."""

    def __init__(self, solver, cfl, probe, checkpoint=20):
        if not isinstance(solver, Solver) or solver.precision == "mixed":
            raise ValueError("the adjoint runs on a float64 Solver")
        self.s = solver
        self.cfl = float(cfl)
        probe = tuple(int(v) for v in probe)
        if solver.dim == 1 and len(probe) == 2:
            probe = (probe[0], 0, probe[1], 1)
        self.probe = probe
        self.K = int(checkpoint)
        L = solver._lib
        _native.check(L.jb_set_probe(solver._h, *self.probe), solver._h, "jb_set_probe")
        _native.check(L.jb_adjoint_reserve(solver._h), solver._h, "jb_adjoint_reserve")
        self.rec_doubles = int(L.jb_record_doubles(solver._h))
        self._lnA = None

    def set_log_A_offset(self, offset):
        """ln A_i offsets (19) applied to the mechanism (None: none)."""
        L = self.s._lib
        if offset is None:
            _native.check(L.jb_set_log_A_offset(self.s._h, None), self.s._h, "jb_set_log_A_offset")
            self._lnA = None
            return
        off = [float(v) for v in torch.as_tensor(offset).detach().cpu().reshape(-1)]
        arr = (ctypes.c_double * len(off))(*off)
        _native.check(L.jb_set_log_A_offset(self.s._h, arr), self.s._h, "jb_set_log_A_offset")
        self._lnA = off

    def run(self, U0, aux0, nsteps):
        """Forward pass: (U, aux, dts, pps, checkpoints) without recording."""
        s, L = self.s, self.s._lib
        dev = U0.device
        dts = torch.empty(nsteps, dtype=torch.float64, device=dev)
        pps = torch.empty(nsteps, dtype=torch.float64, device=dev)
        ckpts = []
        U, aux = U0, aux0
        n = 0
        while n < nsteps:
            k = min(self.K, nsteps - n)
            ckpts.append((U, aux))
            Uo, ao = torch.empty_like(U), torch.empty_like(aux)
            rc = L.jb_advance_ex(s._h, _ptr(U), _ptr(aux), _ptr(Uo), _ptr(ao), 0.0, self.cfl, k, _off(dts, n),
                                 _off(pps, n), None, None, _stream())
            _native.check(rc, s._h, "jb_advance_ex")
            U, aux = Uo, ao
            n += k
        return U, aux, dts, pps, ckpts

    def backward(self, ckpts, nsteps, dts_bar, pps_bar, Ubar=None, Abar=None):
        """Adjoint sweep: returns (Ubar_0, Abar_0, lnA_bar)."""
        s, L = self.s, self.s._lib
        U0 = ckpts[0][0]
        dev = U0.device
        Ub = torch.zeros_like(U0) if Ubar is None else Ubar.clone().contiguous()
        Ab = torch.zeros_like(ckpts[0][1]) if Abar is None else Abar.clone().contiguous()
        lnAb = torch.zeros(19, dtype=torch.float64, device=dev)
        dtb = dts_bar.contiguous() if dts_bar is not None else None
        ppb = pps_bar.contiguous() if pps_bar is not None else None
        scratch_dt = torch.empty(self.K, dtype=torch.float64, device=dev)
        rec = torch.empty((self.K + 1) * self.rec_doubles, dtype=torch.float64, device=dev)
        rslots = torch.empty(self.K * SLOT_DOUBLES, dtype=torch.float64, device=dev)
        Utmp, atmp = torch.empty_like(U0), torch.empty_like(ckpts[0][1])
        for seg in reversed(range(len(ckpts))):
            n0 = seg * self.K
            k = min(self.K, nsteps - n0)
            Uc, ac = ckpts[seg]
            rc = L.jb_advance_ex(s._h, _ptr(Uc), _ptr(ac), _ptr(Utmp), _ptr(atmp), 0.0, self.cfl, k,
                                 _ptr(scratch_dt), None, _ptr(rec), _ptr(rslots), _stream())
            _native.check(rc, s._h, "jb_advance_ex (recompute)")
            for j in reversed(range(k)):
                rc = L.jb_adjoint_step(s._h, _off(rec, j * self.rec_doubles), _off(rslots, j * SLOT_DOUBLES),
                                       self.cfl, _ptr(Ub), _ptr(Ab), _off(dtb, n0 + j), _off(ppb, n0 + j),
                                       _ptr(lnAb), _stream())
                _native.check(rc, s._h, "jb_adjoint_step")
        return Ub, Ab, lnAb

    def state_vjp(self, P, T, Y, Ubar, Abar):
        """T adjoint of the initial-state builder."""
        Tb = torch.empty_like(T)
        rc = self.s._lib.jb_state_from_PTY_vjp(self.s._h, _ptr(P), _ptr(T), _ptr(Y), _ptr(Ubar), _ptr(Abar),
                                              _ptr(Tb), _stream())
        _native.check(rc, self.s._h, "jb_state_from_PTY_vjp")
        return Tb


class _ProbeTrajectory(torch.autograd.Function):
    @staticmethod
    def forward(ctx, T, lnA, traj, P, Y, nsteps):
        traj.set_log_A_offset(lnA)
        Tc = T.detach().contiguous()
        U0, aux0 = traj.s.state_from_PTY(P, Tc, Y)
        _, _, dts, pps, ckpts = traj.run(U0, aux0, nsteps)
        ctx.traj, ctx.nsteps, ctx.ckpts = traj, nsteps, ckpts
        ctx.lnA = None if lnA is None else lnA.detach().clone()
        ctx.save_for_backward(Tc, P, Y)
        return dts, pps

    @staticmethod
    def backward(ctx, dts_bar, pps_bar):
        Tc, P, Y = ctx.saved_tensors
        traj = ctx.traj
        traj.set_log_A_offset(ctx.lnA)
        Ub, Ab, lnAb = traj.backward(ctx.ckpts, ctx.nsteps, dts_bar, pps_bar)
        Tb = traj.state_vjp(P, Tc, Y, Ub, Ab)
        return Tb, (lnAb if ctx.lnA is not None else None), None, None, None, None


def probe_trajectory(traj, P, T, Y, lnA, nsteps):
    """(dts, pps): each step's CFL time step and the probe pressure after it,
    from the state built from (P, T, Y); differentiable in T and lnA."""
    return _ProbeTrajectory.apply(T, lnA, traj, P.contiguous(), Y.contiguous(), int(nsteps))
