"""Torch float64 autograd twin of the reference's 2D and 1D step: the
stand-in for ``jax.grad`` of JANC (``src/janc_v2``), which cannot run here
(no JAX).  1D arrays are (nv, nx) with nv = 11 (solver_1D/*), 2D arrays
(nv, nx, ny) with nv = 12 (solver_2D/*).

TEST INFRASTRUCTURE ONLY.  Only ``tests/`` may import this module; it is the
checker of the hand-written adjoint, never part of the product.

It restates the same functions as ``janc_oracle`` (whose forward is pinned
to the reference's golden vectors) with torch tensors, so that torch's
reverse mode reproduces what ``jax.grad`` of the reference computes:

* ``get_T`` is a custom autograd function with the reference's own VJP
  (model/thermo_model.py:155-190, ``get_T_bwd``): implicit derivatives of
  (gamma, T) with respect to (e, Y) at the converged temperature and no
  derivative with respect to the initial guess;
* ``jnp.nanmax`` (LF alpha, flux_splitting/LF.py) and ``jnp.min`` (CFL,
  set_simulator.py:420-443) split their gradient evenly among tied entries,
  as ``torch.amax`` / ``torch.amin`` do;
* ``jnp.linalg.solve`` (reaction_model.py:159) -> ``torch.linalg.solve``;
  ``jnp.clip`` -> ``torch.clamp``.

Boundaries restated here: the copy types (periodic, slip_wall,
zero_gradient, no_slip_wall), pressure_outlet
(boundary_conditions_2D/pressure_outlet.py:5-66) with the back pressure
``Pb`` a constant (its sub/supersonic switch, a ``jnp.where`` in the
reference, passes gradients to the selected branch only, as
``torch.where`` does), and the rotating-detonation injector of the bottom
side (examples/janc_basic_example2.ipynb ``bottom_boundary`` + ``inj_model``)
with ``Yinj`` a constant (its bisection moves constants through
``jnp.where``, so the Mach number carries no gradient).
"""
import numpy as np
import torch

from . import janc_oracle as jo

TOL, MAX_ITER = jo.TOL, jo.MAX_ITER
_EPS, _C1, _C2, _C3 = 1e-6, 1 / 10, 3 / 5, 3 / 10


class Twin:
    """Mechanism tables as float64 tensors plus the solver configuration."""

    def __init__(self, mech, dx, dy, bc, cfl, device="cpu", Pb=None, Yinj=None, inj_block_p=1.0):
        self.m = mech
        self.dx, self.dy, self.bc, self.cfl = dx, dy, bc, cfl
        self.Pb = Pb
        self.Yinj = None if Yinj is None else torch.as_tensor(np.asarray(Yinj, dtype=np.float64), device=device)
        self.inj_block_p = inj_block_p
        self.dev = device
        t = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=device)
        self.M = t(mech.species_M)
        self.Tcr = t(mech.Tcr)
        for k in ("cp_cof_low", "cp_cof_high", "dcp_cof_low", "dcp_cof_high", "h_cof_low", "h_cof_high",
                  "h_cof_low_chem", "h_cof_high_chem", "s_cof_low", "s_cof_high", "logcof_low",
                  "logcof_high", "A", "B", "EaR", "vf", "vb", "third_body", "is_third_body", "vsum"):
            setattr(self, k, t(getattr(mech, k)))
        self.ns, self.nr = mech.ns, mech.nr


def _ex(v, nd):
    return v.reshape(v.shape + (1,) * nd)


def _seqsum(a):
    s = a[0:1]
    for i in range(1, a.shape[0]):
        s = s + a[i:i + 1]
    return s


def fill_Y(Y):
    return torch.cat([Y, 1.0 - _seqsum(Y)], 0)


def get_R(tw, Y):
    return _seqsum(1 / _ex(tw.M, Y.ndim - 1) * fill_Y(Y))


def _polyval(p, x):
    y = torch.zeros_like(x)
    for c in p:
        y = y * x + c
    return y


def thermo_props(tw, T):
    """Per-species cp, dcp, h (thermo_model.py:100-112); T without the
    leading axis."""
    cp, dcp, h = [], [], []
    for k in range(tw.ns):
        lo = T < tw.Tcr[k]
        cp.append(torch.where(lo, _polyval(tw.cp_cof_low[k], T), _polyval(tw.cp_cof_high[k], T)))
        dcp.append(torch.where(lo, _polyval(tw.dcp_cof_low[k], T), _polyval(tw.dcp_cof_high[k], T)))
        h.append(torch.where(lo, _polyval(tw.h_cof_low[k], T), _polyval(tw.h_cof_high[k], T)))
    return torch.stack(cp), torch.stack(dcp), torch.stack(h)


def get_thermo(tw, T, Y):
    R = get_R(tw, Y)
    Yf = fill_Y(Y)
    cp_i, dcp_i, h_i = thermo_props(tw, T[0])
    cp = _seqsum(cp_i * Yf)
    h = _seqsum(h_i * Yf)
    dcp = _seqsum(dcp_i * Yf)
    return cp, cp / (cp - R), h, R, dcp


class _GetT(torch.autograd.Function):
    """get_T_nasa7 with the reference's custom VJP (thermo_model.py:135-190)."""

    @staticmethod
    def forward(ctx, e, Y, T0, tw):
        with torch.no_grad():
            def eqn(T):
                cp, gamma, h, R, dcp = get_thermo(tw, T, Y)
                return (h - R * T) - e, cp - R, dcp, gamma
            res, d1, d2, gamma = eqn(T0)
            T = T0
            i = 0
            while bool(torch.max(torch.abs(res)) > TOL) and i < MAX_ITER:
                T = T + (-2 * res * d1 / (2 * (d1 * d1) - res * d2))
                res, d1, d2, gamma = eqn(T)
                i += 1
        ctx.save_for_backward(e, Y, T)
        ctx.tw = tw
        return torch.cat([gamma, T], 0)

    @staticmethod
    def backward(ctx, g):
        e, Y, T = ctx.saved_tensors
        tw = ctx.tw
        nd = T.ndim - 1
        cp, _, h, R, dcp = get_thermo(tw, T, Y)
        cv = cp - R
        dT_de = 1 / cv
        dgamma_dT = (dcp * cv - dcp * cp) / (cv ** 2)
        cp_i, _, h_i = thermo_props(tw, T[0])
        e_i = h_i - 1 / _ex(tw.M, nd) * T
        dT_dY = (-e_i[0:-1] + e_i[-1:]) / cv
        dR_dY = _ex(1 / tw.M[0:-1] - 1 / tw.M[-1:], nd)
        dcp_dY = cp_i[0:-1] - cp_i[-1:]
        dcv_dY = dcp_dY - dR_dY
        dgamma_dY = dgamma_dT * dT_dY + (dcp_dY * cv - dcv_dY * cp) / (cv ** 2)
        gg, gT = g[0:1], g[1:2]
        return gg * dgamma_dT * dT_de + gT * dT_de, gg * dgamma_dY + gT * dT_dY, None, None


def _nY(U):
    return 3 if U.ndim == 2 else 4


def update_aux(tw, U, aux):
    """solver_2D/aux_func.py:21-29, solver_1D/aux_func.py:21-28"""
    rho = U[0:1]
    u = U[1:2] / rho
    if U.ndim == 2:
        e = U[2:3] / rho - 0.5 * (u ** 2)
    else:
        v = U[2:3] / rho
        e = U[3:4] / rho - 0.5 * (u ** 2 + v ** 2)
    Y = U[_nY(U):] / rho
    return _GetT.apply(e, Y, aux[1:2], tw)


def prims(tw, U, aux):
    """U_to_prim (v = 0 in 1D)"""
    gamma, T = aux[0:1], aux[1:2]
    rho = U[0:1]
    u = U[1:2] / rho
    v = U[2:3] / rho if U.ndim == 3 else torch.zeros_like(u)
    Y = U[_nY(U):] / rho
    R = get_R(tw, Y)
    p = rho * R * T
    a = torch.sqrt(gamma * p / rho)
    return rho, u, v, Y, p, a


# ------------------------------------------------------------------ chemistry
def get_gibbs(tw, T):
    out = []
    for k in range(tw.nr):
        lo = T < tw.Tcr[k]
        h = torch.where(lo, _polyval(tw.h_cof_low_chem[k], T), _polyval(tw.h_cof_high_chem[k], T))
        lt = torch.log(tw.m.nondim.T0 * T)
        s = torch.where(lo, _polyval(tw.s_cof_low[k], T) + tw.logcof_low[k] * lt,
                        _polyval(tw.s_cof_high[k], T) + tw.logcof_high[k] * lt)
        out.append(s - h / T)
    return torch.stack(out)


def reaction_source_terms(tw, U, aux, dt, lnA_offset=None):
    """reaction_model.py:91-193; lnA_offset (19) scales A_i by exp()."""
    nd = U.ndim - 1
    nY = _nY(U)
    nr, nreac = tw.nr, tw.A.shape[0]
    rho = U[0:1]
    Y = fill_Y(U[nY:] / rho)
    rhoY = rho * Y
    T = aux[1:2]
    X = rhoY / _ex(tw.M, nd)
    g = get_gibbs(tw, T[0])
    Xc = torch.clamp(X, min=1e-50)
    log_X = torch.log(Xc[0:nr])
    A = tw.A if lnA_offset is None else tw.A * torch.exp(lnA_offset)
    kf_l, kb_l, M_l = [], [], []
    for i in range(nreac):
        vf_i, vb_i = _ex(tw.vf[i], nd), _ex(tw.vb[i], nd)
        kf_i = A[i] * torch.pow(T, tw.B[i]) * torch.exp(-tw.EaR[i] / T)
        Msum = _seqsum(_ex(tw.third_body[i], nd) * X)
        Msum = tw.is_third_body[i] * Msum + (1 - tw.is_third_body[i])
        kf = kf_i * torch.exp(_seqsum(vf_i * log_X))
        kb = kf_i / (torch.exp(_seqsum((vb_i - vf_i) * g)) * ((101325 / tw.m.nondim.P0 / T) ** tw.vsum[i])) \
            * torch.exp(_seqsum(vb_i * log_X))
        kf_l.append(kf)
        kb_l.append(kb)
        M_l.append(Msum)
    w, Jrows = [], []
    for k in range(nr):
        Mk = tw.M[k]
        w.append(Mk * _seqsum(torch.stack([(tw.vb[i, k] - tw.vf[i, k]) * M_l[i] * (kf_l[i] - kb_l[i])
                                           for i in range(nreac)]))[0, 0])
        row = []
        for n in range(nr):
            Mn = tw.M[n]
            Xn = Xc[n][None]
            tn = [(tw.vb[i, k] - tw.vf[i, k]) * (kf_l[i] - kb_l[i]) * (tw.third_body[i, n] / Mn)
                  + 1 / (Mn * Xn) * (tw.vb[i, k] - tw.vf[i, k]) * M_l[i]
                  * (tw.vf[i, n] * kf_l[i] - tw.vb[i, n] * kb_l[i]) for i in range(nreac)]
            row.append(Mk * _seqsum(torch.stack(tn))[0, 0])
        Jrows.append(torch.stack(row))
    S = torch.movedim(torch.stack(w), 0, -1)[..., None]
    J = torch.stack(Jrows)                                   # (nr, nr, ...)
    DSDU = torch.movedim(torch.movedim(J, 0, -1), 0, -1)     # (..., nr, nr)
    Amat = torch.eye(nr, dtype=U.dtype, device=U.device) / dt - DSDU
    x = torch.linalg.solve(Amat, S)
    drhoY = torch.movedim(x[..., 0], -1, 0)
    dY = drhoY / rho
    dY = torch.clamp(dY, -Y[0:-1], 1 - Y[0:-1])
    return torch.cat([torch.zeros_like(U[:nY]), rho * dY], 0)


# ------------------------------------------------------------------ flux
def _pressure_outlet_state(tw, state, gamma, T, normal_vel):
    """boundary_conditions_{1D,2D}/pressure_outlet.py:5-22 (janc_oracle's
    _pressure_outlet_state in torch)."""
    two_d = state.ndim == 3
    rho = state[0:1]
    u = state[1:2] / rho
    v = state[2:3] / rho if two_d else None
    Y = state[_nY(state):] / rho
    R = get_R(tw, Y)
    p = rho * (R * T)
    a = torch.sqrt(gamma * p / rho)
    mask = normal_vel / a < 1
    Pb = tw.Pb
    rho_c = torch.where(mask, Pb / (p / rho), rho)
    p_c = torch.where(mask, Pb * torch.ones_like(p), p)
    T_c = torch.where(mask, p_c / (rho_c * R), T)
    _, gamma_c, h_c, _, _ = get_thermo(tw, T_c, Y)
    if two_d:
        Ub = torch.cat([rho_c, rho_c * u, rho_c * v, rho_c * h_c - p_c + 0.5 * rho_c * (u ** 2 + v ** 2),
                        rho_c * Y], 0)
    else:
        Ub = torch.cat([rho_c, rho_c * u, rho_c * h_c - p_c + 0.5 * rho_c * (u ** 2), rho_c * Y], 0)
    return Ub, torch.cat([gamma_c, T_c], 0)


def _inj_model(tw, p, Y_inj):
    """inj_model of examples/janc_basic_example2.ipynb (janc_oracle's
    inj_model in torch)."""
    A1, A3 = 1, 5
    A2 = A3 - A1
    R = get_R(tw, Y_inj)
    gamma = 1.29
    C0 = torch.sqrt(gamma * R * 1.0)
    P3 = p
    M1 = torch.zeros_like(p)
    M2 = torch.ones_like(p)
    for _ in range(20):
        M = 0.5 * (M1 + M2)
        P1 = 1.0 * (1 + (gamma - 1) / 2 * M ** 2) ** (-gamma / (gamma - 1))
        V1 = M * (1 + (gamma - 1) / 2 * M ** 2) ** (-0.5) * C0
        MFC = A1 * 1.0 / np.sqrt(1.0) * torch.sqrt(gamma / R) * M * (1 + (gamma - 1) / 2 * M ** 2) ** (
            -(gamma + 1) / 2 / (gamma - 1))
        A = 0.5
        B = gamma / (gamma - 1) * P3 * A3 / MFC
        C = -gamma / (gamma - 1) * R * 1.0
        V3 = (-B + torch.sqrt(B ** 2 - 4 * A * C)) / (2 * A)
        P2 = (MFC * (V3 - V1) - P1 * A1 + P3 * A3) / A2
        M2 = torch.where(P2 >= P1, M, M2)
        M1 = torch.where(P2 < P1, M, M1)
    rho_c = MFC / V3 / A3
    v_c = V3
    T_c = p / (R * rho_c)
    _, gamma_c, h_c, _, _ = get_thermo(tw, T_c, Y_inj)
    return v_c, T_c, h_c, gamma_c


def _injector_state(tw, state, aux, Yinj):
    """bottom_boundary of examples/janc_basic_example2.ipynb on the first
    interior row (janc_oracle's _injector_state in torch)."""
    rho, u, v, Y, p, a = prims(tw, state, aux)
    T = aux[1:2]
    gamma = aux[0:1]
    _, _, h, R, _ = get_thermo(tw, T, Y)
    u_inj = torch.zeros_like(u)
    v_inj, T_inj, h_inj, g_inj = _inj_model(tw, p, Yinj)
    R_inj = get_R(tw, Yinj)
    rho_inj = p / (R_inj * T_inj)
    blk = p >= tw.inj_block_p
    rho_c = torch.where(blk, rho, rho_inj)
    u_c = torch.where(blk, u, u_inj)
    v_c = torch.where(blk, -v, v_inj)
    T_c = torch.where(blk, T, T_inj)
    p_c = p
    h_c = torch.where(blk, h, h_inj)
    Y_c = torch.where(blk.expand(Yinj.shape[0], -1, -1), Y, Yinj)
    g_c = torch.where(blk, gamma, g_inj)
    Ub = torch.cat([rho_c, rho_c * u_c, rho_c * v_c,
                    rho_c * h_c - p_c + 0.5 * rho_c * (u_c ** 2 + v_c ** 2), rho_c * Y_c], 0)
    return Ub, torch.cat([g_c, T_c], 0)


def _bc_side(tw, kind, side, Ub, auxb):
    ax = 1 if side in "LR" else 2
    lo = side in "LB"
    shp = (-1,) + (1,) * (Ub.ndim - 1)

    def take(a, j):
        return a.narrow(ax, j if j >= 0 else a.shape[ax] + j, 1)

    if kind in ("zero_gradient", "no_slip_wall"):
        order = [2, 1, 0] if lo else [-1, -2, -3]
        U = torch.cat([take(Ub, j) for j in order], ax)
        A = torch.cat([take(auxb, j) for j in order], ax)
        if kind == "no_slip_wall":
            sgn = torch.ones(Ub.shape[0], dtype=Ub.dtype, device=Ub.device)
            sgn[1:3 if Ub.ndim == 3 else 2] = -1
            U = U * sgn.reshape(shp)
        return U, A
    if kind == "slip_wall":
        j = 0 if lo else -1
        U = torch.cat([take(Ub, j)] * 3, ax)
        A = torch.cat([take(auxb, j)] * 3, ax)
        sgn = torch.ones(Ub.shape[0], dtype=Ub.dtype, device=Ub.device)
        sgn[1 if side in "LR" else 2] = -1
        return U * sgn.reshape(shp), A
    if kind == "rdc_injector":
        assert side == "B" and Ub.ndim == 3
        st, au = Ub[:, :, 0:1], auxb[:, :, 0:1]
        Yinj = tw.Yinj
        if Yinj.ndim == 1:
            Yinj = Yinj[:, None, None].expand(-1, Ub.shape[1], 1)
        Us, As = _injector_state(tw, st, au, Yinj)
        return torch.cat([Us] * 3, 2), torch.cat([As] * 3, 2)
    if kind == "pressure_outlet":
        j = 0 if lo else -1
        st, ga, Tt = take(Ub, j), take(auxb[0:1], j), take(auxb[1:2], j)
        mom = 1 if side in "LR" else 2
        nv = st[mom:mom + 1] / st[0:1]
        if lo:
            nv = -nv
        Us, As = _pressure_outlet_state(tw, st, ga, Tt, nv)
        return torch.cat([Us] * 3, ax), torch.cat([As] * 3, ax)
    raise KeyError(f"the twin does not restate the {kind} boundary")


def boundary_conditions(tw, U, aux):
    if U.ndim == 2:  # boundary.py:120-126 (1D): periodic pad, then left, right
        f = torch.cat([U, aux], 0)
        f = torch.cat([f[:, -4:-3], f[:, -3:-2], f[:, -2:-1], f, f[:, 1:2], f[:, 2:3], f[:, 3:4]], 1)
        Up, Ap = f[:-2].clone(), f[-2:].clone()
        for s, key, src, dst in (("L", "left_boundary", slice(3, 6), slice(0, 3)),
                                 ("R", "right_boundary", slice(-6, -3), slice(-3, None))):
            kind = tw.bc[key]
            if kind == "periodic":
                continue
            Ug, Ag = _bc_side(tw, kind, s, Up[:, src].clone(), Ap[:, src].clone())
            Up[:, dst] = Ug
            Ap[:, dst] = Ag
        return Up, Ap
    f = torch.cat([U, aux], 0)
    f = torch.cat([f[:, -4:-3], f[:, -3:-2], f[:, -2:-1], f, f[:, 1:2], f[:, 2:3], f[:, 3:4]], 1)
    f = torch.cat([f[:, :, -4:-3], f[:, :, -3:-2], f[:, :, -2:-1], f, f[:, :, 1:2], f[:, :, 2:3], f[:, :, 3:4]], 2)
    Up, Ap = f[:-2].clone(), f[-2:].clone()
    sl = {"L": (slice(None), slice(3, 6), slice(3, -3)), "R": (slice(None), slice(-6, -3), slice(3, -3)),
          "B": (slice(None), slice(3, -3), slice(3, 6)), "T": (slice(None), slice(3, -3), slice(-6, -3))}
    dst = {"L": (slice(None), slice(0, 3), slice(3, -3)), "R": (slice(None), slice(-3, None), slice(3, -3)),
           "B": (slice(None), slice(3, -3), slice(0, 3)), "T": (slice(None), slice(3, -3), slice(-3, None))}
    for s, key in (("L", "left_boundary"), ("R", "right_boundary"), ("B", "bottom_boundary"),
                   ("T", "top_boundary")):
        kind = tw.bc[key]
        if kind == "periodic":
            continue
        # the side reads copies: later sides write into Up / Ap in place
        Ug, Ag = _bc_side(tw, kind, s, Up[sl[s]].clone(), Ap[sl[s]].clone())
        Up[dst[s]] = Ug
        Ap[dst[s]] = Ag
    return Up, Ap


def _sq(x):
    return x * x


def _weno_L(fjm2, fjm1, fj, fjp1, fjp2):
    IS1 = 1 / 4 * _sq(fjm2 - 4 * fjm1 + 3 * fj) + 13 / 12 * _sq(fjm2 - 2 * fjm1 + fj)
    IS2 = 1 / 4 * _sq(fjm1 - fjp1) + 13 / 12 * _sq(fjm1 - 2 * fj + fjp1)
    IS3 = 1 / 4 * _sq(3 * fj - 4 * fjp1 + fjp2) + 13 / 12 * _sq(fj - 2 * fjp1 + fjp2)
    a1 = _C1 / _sq(_EPS + IS1)
    a2 = _C2 / _sq(_EPS + IS2)
    a3 = _C3 / _sq(_EPS + IS3)
    s = a1 + a2 + a3
    q1 = 1 / 3 * fjm2 - 7 / 6 * fjm1 + 11 / 6 * fj
    q2 = -1 / 6 * fjm1 + 5 / 6 * fj + 1 / 3 * fjp1
    q3 = 1 / 3 * fj + 5 / 6 * fjp1 - 1 / 6 * fjp2
    return a1 / s * q1 + a2 / s * q2 + a3 / s * q3


def _weno_R(fjm2, fjm1, fj, fjp1, fjp2):
    return _weno_L(fjp2, fjp1, fj, fjm1, fjm2)


def _faces(q, axis, lo, hi):
    idx = [slice(None)] * 3
    idx[axis] = slice(lo, hi)
    idx[3 - axis] = slice(3, -3)
    return q[tuple(idx)]


def total_flux(tw, Up, Ap):
    if Up.ndim == 2:  # solver_1D/flux.py flux_splitting with LF and WENO5-JS
        rho, u, v, Y, p, a = prims(tw, Up, Ap)
        um = torch.amax(torch.abs(u) + a)
        F = torch.cat([rho * u, rho * u ** 2 + p, u * (Up[2:3] + p), rho * u * Y], 0)
        Fp, Fm = 0.5 * (F + um * Up), 0.5 * (F - um * Up)
        n = Up.shape[1]
        L = _weno_L(*[Fp[:, k:n - 5 + k] for k in range(5)])
        R = _weno_R(*[Fm[:, 1 + k:n - 4 + k] for k in range(5)])
        Fx = L + R
        return -(Fx[:, 1:] - Fx[:, :-1]) / tw.dx
    rho, u, v, Y, p, a = prims(tw, Up, Ap)
    rhoE = Up[3:4]
    um = torch.amax(torch.abs(u) + a)
    vm = torch.amax(torch.abs(v) + a)
    F = torch.cat([rho * u, rho * u ** 2 + p, rho * u * v, u * (rhoE + p), rho * u * Y], 0)
    G = torch.cat([rho * v, rho * u * v, rho * v ** 2 + p, v * (rhoE + p), rho * v * Y], 0)
    Fp, Fm = 0.5 * (F + um * Up), 0.5 * (F - um * Up)
    Gp, Gm = 0.5 * (G + vm * Up), 0.5 * (G - vm * Up)
    n = Up.shape[1]

    def face(Hp, Hm, axis):
        n = Hp.shape[axis]
        L = _weno_L(*[_faces(Hp, axis, k, n - 5 + k) for k in range(5)])
        R = _weno_R(*[_faces(Hm, axis, 1 + k, n - 4 + k) for k in range(5)])
        return L + R
    Fx = face(Fp, Fm, 1)
    Gy = face(Gp, Gm, 2)
    del n
    dF = Fx[:, 1:, :] - Fx[:, :-1, :]
    dG = Gy[:, :, 1:] - Gy[:, :, :-1]
    return -(dF / tw.dx + dG / tw.dy)


def flux_func(tw, U, aux, dt):
    Up, Ap = boundary_conditions(tw, U, aux)
    return dt * total_flux(tw, Up, Ap)


def cfl_dt(tw, U, aux):
    _, u, v, _, _, a = prims(tw, U, aux)
    sx = torch.abs(u) + a
    if U.ndim == 2:  # CFL_1D
        return tw.cfl * torch.amin(tw.dx / sx)
    sy = torch.abs(v) + a
    return tw.cfl * torch.amin(1 / (sx / tw.dx + sy / tw.dy))


def advance_one_step(tw, U, aux, dt, lnA_offset=None):
    U1 = U + flux_func(tw, U, aux, dt)
    aux1 = update_aux(tw, U1, aux)
    U2 = 3 / 4 * U + 1 / 4 * (U1 + flux_func(tw, U1, aux1, dt))
    aux2 = update_aux(tw, U2, aux1)
    U3 = 1 / 3 * U + 2 / 3 * (U2 + flux_func(tw, U2, aux2, dt))
    aux3 = update_aux(tw, U3, aux2)
    U4 = U3 + reaction_source_terms(tw, U3, aux3, dt, lnA_offset)
    aux4 = update_aux(tw, U4, aux3)
    return U4, aux4


def state_from_PTY(tw, P, T, Y):
    _, gamma, h, R, _ = get_thermo(tw, T, Y)
    rho = P / (R * T)
    E = rho * h - P
    z = torch.zeros_like(T)
    if T.ndim == 2:
        U = torch.cat([rho, rho * z, E, rho * Y], 0)
    else:
        U = torch.cat([rho, rho * z, rho * z, E, rho * Y], 0)
    return U, torch.cat([gamma, T], 0)


def probe_pressure(tw, U, aux, probe):
    """Mean pressure over the probe cells (x0, y0, wx, wy); 1D: (x0, 0, wx, 1)."""
    x0, y0, wx, wy = probe
    _, _, _, _, p, _ = prims(tw, U, aux)
    if U.ndim == 2:
        return p[0, x0:x0 + wx].mean()
    return p[0, x0:x0 + wx, y0:y0 + wy].mean()


def trajectory_loss(tw, P, T, Y, nsteps, probe, lnA_offset=None):
    """L = sum_n dt_n * mean probe pressure after step n, from the state
    built from (P, T, Y); returns (L, dts, probe pressures)."""
    U, aux = state_from_PTY(tw, P, T, Y)
    L = 0.0
    dts, pps = [], []
    for _ in range(nsteps):
        dt = cfl_dt(tw, U, aux)
        U, aux = advance_one_step(tw, U, aux, dt, lnA_offset)
        pp = probe_pressure(tw, U, aux, probe)
        L = L + dt * pp
        dts.append(dt)
        pps.append(pp)
    return L, torch.stack(dts), torch.stack(pps)
