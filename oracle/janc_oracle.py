"""CPU oracle: a NumPy float64 restatement of JANC's per-step reacting-flow
path (``src/janc_v2`` of luofx23/JANC).

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import this module; the product
(``janc_b200``) never calls it.

Every function follows the reference array-for-array and keeps its operation
order (Python left-to-right evaluation of the same expressions), so on the
reference's golden vectors it agrees to the last bit except where libm
``exp``/``log``/``pow`` or LAPACK's pivoted solve order differ.  Arrays use the
reference layout: ``U`` is ``(nv, nx)`` in 1D and ``(nv, nx, ny)`` in 2D with
``nv = 3 + 8`` resp. ``4 + 8``; ``aux`` is ``(2, ...)`` = ``[gamma, T]``.

Cited reference files (paths inside the JANC repository):
  preprocess/load.py, preprocess/nondim.py, model/thermo_model.py,
  model/reaction_model.py, solver_{1D,2D}/aux_func.py,
  solver_{1D,2D}/flux.py, solver_{1D,2D}/flux_splitting/LF.py,
  solver_{1D,2D}/reconstruction/WENO5_JS.py, boundary/boundary.py,
  boundary/boundary_padding.py, boundary/boundary_conditions_{1D,2D}/*.py,
  simulation/time_step/TVD_RK3.py, simulation/set_simulator.py,
  examples/janc_basic_example2.ipynb (rotating-detonation injector).
"""
from dataclasses import dataclass, field

import numpy as np
import yaml

RG = 8.314463  # preprocess/nondim.py:3
MAX_ITER = 5   # model/thermo_model.py:17
TOL = 5e-9     # model/thermo_model.py:18
ATOMIC_WEIGHT = {"H": 1.008, "He": 4.002602, "C": 12.011, "N": 14.007, "O": 15.999, "Ar": 39.95}
EA_TO_J_PER_KMOL = {"cal/mol": 4184.0, "kcal/mol": 4184000.0, "J/mol": 1000.0,
                    "kJ/mol": 1.0e6, "J/kmol": 1.0}


# --------------------------------------------------------------------------
# reference scales  (preprocess/nondim.py:14-25)
# --------------------------------------------------------------------------
@dataclass
class Nondim:
    P0: float = 1.0
    T0: float = 1.0
    R0: float = 1.0
    x0: float = 1.0

    @property
    def rho0(self):
        return self.P0 / (self.R0 * self.T0)

    @property
    def M0(self):
        return RG / self.R0

    @property
    def e0(self):
        return self.P0 / self.rho0

    @property
    def u0(self):
        return np.sqrt(self.P0 / self.rho0)

    @property
    def t0(self):
        return self.x0 / self.u0


# --------------------------------------------------------------------------
# mechanism tables
# --------------------------------------------------------------------------
@dataclass
class Mech:
    species: list
    nondim: Nondim
    species_M: np.ndarray
    Tcr: np.ndarray
    cp_cof_low: np.ndarray
    cp_cof_high: np.ndarray
    dcp_cof_low: np.ndarray
    dcp_cof_high: np.ndarray
    h_cof_low: np.ndarray
    h_cof_high: np.ndarray
    h_cof_low_chem: np.ndarray
    h_cof_high_chem: np.ndarray
    s_cof_low: np.ndarray
    s_cof_high: np.ndarray
    logcof_low: np.ndarray
    logcof_high: np.ndarray
    A: np.ndarray
    B: np.ndarray
    EaR: np.ndarray
    vf: np.ndarray
    vb: np.ndarray
    third_body: np.ndarray
    is_third_body: np.ndarray
    vsum: np.ndarray
    extra: dict = field(default_factory=dict)

    @property
    def ns(self):
        return len(self.species)

    @property
    def nr(self):
        return self.vf.shape[1]

    def tables(self):
        keys = ["species_M", "Tcr", "cp_cof_low", "cp_cof_high", "dcp_cof_low", "dcp_cof_high",
                "h_cof_low", "h_cof_high", "h_cof_low_chem", "h_cof_high_chem", "s_cof_low",
                "s_cof_high", "logcof_low", "logcof_high", "A", "B", "EaR", "vf", "vb",
                "third_body", "is_third_body", "vsum"]
        return {k: getattr(self, k) for k in keys}


def _parse_side(side):
    out, has_m = {}, False
    for tok in side.split(" + "):
        tok = tok.strip()
        if tok == "M":
            has_m = True
            continue
        parts = tok.split()
        if len(parts) == 2:
            nu, sp = float(parts[0]), parts[1]
        else:
            nu, sp = 1.0, tok
        out[sp] = out.get(sp, 0.0) + nu
    return out, has_m


def load_mechanism(path, nondim=None):
    """Cantera-style YAML -> the reference's constant tables.

    Restates ``preprocess/load.py:8-135`` (``read_reaction_mechanism`` and
    ``get_cantera_coeffs``) together with the Cantera 3.x conventions it relies
    on (A to SI-kmol by (1e-3)**(order-1) for cm/mol input, Ea to J/kmol by
    4184 per cal/mol, NASA7 coefficient packing, IUPAC atomic weights).
    """
    nd = nondim if isinstance(nondim, Nondim) else (Nondim(**nondim) if nondim else Nondim())
    with open(path) as f:
        doc = yaml.safe_load(f)
    units = doc.get("units", {})
    cgs = (units.get("length", "m"), units.get("quantity", "kmol")) == ("cm", "mol")
    ea_f = EA_TO_J_PER_KMOL[units.get("activation-energy", "J/kmol")]
    phase = doc["phases"][0]
    species = list(phase["species"])
    elements = list(phase["elements"])
    sp_by = {s["name"]: s for s in doc["species"]}
    ns = len(species)
    # --- species thermo (load.py:91-135)
    Tcr, low, high, MW = [], [], [], []
    for name in species:
        s = sp_by[name]
        w = 0.0
        for el in elements:
            if el in s["composition"]:
                w += s["composition"][el] * ATOMIC_WEIGHT[el]
        MW.append(w)
        th = s["thermo"]
        Tcr.append(th["temperature-ranges"][1])
        low.append(th["data"][0])
        high.append(th["data"][1])
    scale = np.array([[1, nd.T0, nd.T0 ** 2, nd.T0 ** 3, nd.T0 ** 4, 1 / nd.T0, 1]])
    coeffs_low = np.array(low, dtype=np.float64) * scale
    coeffs_high = np.array(high, dtype=np.float64) * scale
    species_M = np.array(MW) / (1000 * nd.M0)
    Tcr = np.array(Tcr, dtype=np.float64) / nd.T0
    cp_cof_low = np.flip(coeffs_low[:, 0:5], axis=1) / species_M[:, None]
    cp_cof_high = np.flip(coeffs_high[:, 0:5], axis=1) / species_M[:, None]
    dcp_cof_low = cp_cof_low[:, 0:-1] * np.array([[4, 3, 2, 1]])
    dcp_cof_high = cp_cof_high[:, 0:-1] * np.array([[4, 3, 2, 1]])
    hw = np.array([[1 / 5, 1 / 4, 1 / 3, 1 / 2, 1, 1]])
    h_cof_low = np.flip(np.roll(coeffs_low[:, 0:6], 1, axis=1), axis=1) * hw / species_M[:, None]
    h_cof_high = np.flip(np.roll(coeffs_high[:, 0:6], 1, axis=1), axis=1) * hw / species_M[:, None]
    h_cof_low_chem = np.flip(np.roll(coeffs_low[:, 0:6], 1, axis=1), axis=1) * hw
    h_cof_high_chem = np.flip(np.roll(coeffs_high[:, 0:6], 1, axis=1), axis=1) * hw
    sw = np.array([[1 / 4, 1 / 3, 1 / 2, 1, 1]])
    s_cof_low = np.flip(np.concatenate([coeffs_low[:, -1:], coeffs_low[:, 1:5]], axis=1), axis=1) * sw
    s_cof_high = np.flip(np.concatenate([coeffs_high[:, -1:], coeffs_high[:, 1:5]], axis=1), axis=1) * sw
    logcof_low = coeffs_low[:, 0]
    logcof_high = coeffs_high[:, 0]
    # --- reactions (load.py:8-88)
    rxns = doc.get("reactions", [])
    nreac = len(rxns)
    vf = np.zeros((nreac, ns))
    vb = np.zeros((nreac, ns))
    A, B, Ea = [], [], []
    tb = np.zeros((nreac, ns))
    is_tb = np.zeros(nreac)
    idx = {n: i for i, n in enumerate(species)}
    for i, r in enumerate(rxns):
        eq = r["equation"]
        for arrow in ("<=>", "=>", "="):
            if arrow in eq:
                lhs, rhs = eq.split(arrow)
                break
        reac, m_l = _parse_side(lhs)
        prod, _ = _parse_side(rhs)
        three = r.get("type", "elementary") == "three-body" or m_l
        for sp, nu in reac.items():
            vf[i, idx[sp]] = nu
        for sp, nu in prod.items():
            vb[i, idx[sp]] = nu
        order = sum(reac.values())
        if three:
            order += 1
            eff = r.get("efficiencies", {})
            for j, sp in enumerate(species):
                tb[i, j] = eff.get(sp, 1.0)
        is_tb[i] = 1.0 * bool(np.any(tb[i, :] > 0))
        rc = r["rate-constant"]
        a_si = float(rc["A"]) * (1.0e-3) ** (order - 1) if cgs else float(rc["A"])
        A.append(a_si * ((1e-3) ** (order - 1)))
        B.append(float(rc["b"]))
        Ea.append(float(rc["Ea"]) * ea_f / 1000)
    nonzero = np.any(vf + vb != 0, axis=0)
    vf = vf[:, nonzero]
    vb = vb[:, nonzero]
    vf_sum = np.sum(vf, axis=1)
    vb_sum = np.sum(vb, axis=1)
    A = np.array(A)
    B = np.array(B)
    Ea = np.array(Ea)
    A = (nd.t0 / nd.rho0) * (nd.T0 ** B) * ((nd.rho0 / nd.M0) ** vf_sum) * nd.M0 * A
    EaR = Ea / (nd.e0 * nd.M0)
    tb = tb * (nd.rho0 / nd.M0)
    return Mech(species, nd, species_M, Tcr, cp_cof_low, cp_cof_high, dcp_cof_low, dcp_cof_high,
                h_cof_low, h_cof_high, h_cof_low_chem, h_cof_high_chem, s_cof_low, s_cof_high,
                logcof_low, logcof_high, A, B, EaR, vf, vb, tb, is_tb, vb_sum - vf_sum,
                extra={"MW": np.array(MW)})


def _ex(v, nd):
    """Broadcast a per-species column over ``nd`` spatial axes."""
    return v.reshape(v.shape + (1,) * nd)


# --------------------------------------------------------------------------
# thermo  (model/thermo_model.py)
# --------------------------------------------------------------------------
def _seqsum(a):
    """Sum over the leading axis in index order, keeping it (size 1).  This is
    the order NumPy uses for a C-contiguous array; making it explicit keeps
    the oracle independent of the caller's memory layout (NumPy sums a
    Fortran-ordered array pairwise)."""
    s = a[0:1]
    for i in range(1, a.shape[0]):
        s = s + a[i:i + 1]
    return s


def fill_Y(Y):
    """thermo_model.py:80-82"""
    return np.concatenate([Y, 1.0 - _seqsum(Y)], axis=0)


def get_R(m, Y):
    """thermo_model.py:87-92"""
    Yf = fill_Y(Y)
    return _seqsum(1 / _ex(m.species_M, Y.ndim - 1) * Yf)


def _polyval(p, x):
    y = np.zeros_like(x)
    for c in p:
        y = y * x + c
    return y


def get_thermo_properties(m, T):
    """thermo_model.py:100-112 (T without the leading axis)."""
    cp, dcp, h = [], [], []
    for k in range(m.ns):
        mask = T < m.Tcr[k]
        cp.append(np.where(mask, _polyval(m.cp_cof_low[k], T), _polyval(m.cp_cof_high[k], T)))
        dcp.append(np.where(mask, _polyval(m.dcp_cof_low[k], T), _polyval(m.dcp_cof_high[k], T)))
        h.append(np.where(mask, _polyval(m.h_cof_low[k], T), _polyval(m.h_cof_high[k], T)))
    return np.stack(cp), np.stack(dcp), np.stack(h)


def get_thermo(m, T, Y):
    """thermo_model.py:115-126 -> (cp, gamma, h, R, dcp)"""
    R = get_R(m, Y)
    Yf = fill_Y(Y)
    cp_i, dcp_i, h_i = get_thermo_properties(m, T[0])
    cp = _seqsum(cp_i * Yf)
    h = _seqsum(h_i * Yf)
    dcp = _seqsum(dcp_i * Yf)
    gamma = cp / (cp - R)
    return cp, gamma, h, R, dcp


def _e_eqn(m, T, e, Y):
    """thermo_model.py:128-133"""
    cp, gamma, h, R, dcp = get_thermo(m, T, Y)
    res = (h - R * T) - e
    return res, cp - R, dcp, gamma


def get_T(m, e, Y, T0, return_iters=False):
    """Halley solve with the reference's global stop test
    (thermo_model.py:135-153): iterate while max|res| > tol and i < 5."""
    res, d1, d2, gamma = _e_eqn(m, T0, e, Y)
    T = T0
    i = 0
    while (np.max(np.abs(res)) > TOL) and (i < MAX_ITER):
        dT = -2 * res * d1 / (2 * (d1 * d1) - res * d2)
        T = T + dT
        res, d1, d2, gamma = _e_eqn(m, T, e, Y)
        i += 1
    out = np.concatenate([gamma, T], axis=0)
    return (out, i) if return_iters else out


# --------------------------------------------------------------------------
# conserved <-> primitive  (solver_{1D,2D}/aux_func.py)
# --------------------------------------------------------------------------
def nY_of(U):
    return 3 if U.ndim == 2 else 4


def update_aux(m, U, aux, return_iters=False):
    """aux_func.py:21-28 (1D) / 21-29 (2D)"""
    rho = U[0:1]
    u = U[1:2] / rho
    if U.ndim == 2:
        e = U[2:3] / rho - 0.5 * (u ** 2)
        Y = U[3:] / rho
    else:
        v = U[2:3] / rho
        e = U[3:4] / rho - 0.5 * (u ** 2 + v ** 2)
        Y = U[4:] / rho
    r = get_T(m, e, Y, aux[1:2], return_iters)
    if return_iters:
        out, it = r
        return out, it
    return r


def U_to_prim(m, U, aux):
    """aux_func.py:39-50 (1D) / 39-51 (2D); returns (rho, u, [v,] Y, p, a)"""
    gamma, T = aux[0:1], aux[1:2]
    rho = U[0:1]
    u = U[1:2] / rho
    if U.ndim == 2:
        Y = U[3:] / rho
        R = get_R(m, Y)
        p = rho * R * T
        a = np.sqrt(gamma * p / rho)
        return rho, u, Y, p, a
    v = U[2:3] / rho
    Y = U[4:] / rho
    R = get_R(m, Y)
    p = rho * R * T
    a = np.sqrt(gamma * p / rho)
    return rho, u, v, Y, p, a


# --------------------------------------------------------------------------
# chemistry  (model/reaction_model.py)
# --------------------------------------------------------------------------
def get_gibbs(m, T):
    """reaction_model.py:78-89 for the nr reactive species; T without the
    leading axis."""
    out = []
    for k in range(m.nr):
        mask = T < m.Tcr[k]
        h = np.where(mask, _polyval(m.h_cof_low_chem[k], T), _polyval(m.h_cof_high_chem[k], T))
        s = np.where(mask, _polyval(m.s_cof_low[k], T) + m.logcof_low[k] * np.log((m.nondim.T0) * T),
                     _polyval(m.s_cof_high[k], T) + m.logcof_high[k] * np.log((m.nondim.T0) * T))
        out.append(s - h / T)
    return np.stack(out)


def construct_matrix_equation(m, T, X, dt):
    """reaction_model.py:91-159: rates, analytic Jacobian and the 8x8 solve.
    T is (1, ...), X is (ns, ...); returns drhoY (nr, ...)."""
    nr, nreac = m.nr, len(m.A)
    nd = T.ndim - 1
    g = get_gibbs(m, T[0])                       # (nr, ...)
    Xc = np.clip(X, 1e-50, None)
    log_X = np.log(Xc[0:nr])
    kf_l, kb_l, M_l = [], [], []
    for i in range(nreac):
        vf_i = _ex(m.vf[i], nd)
        vb_i = _ex(m.vb[i], nd)
        aij = _ex(m.third_body[i], nd)
        kf_i = m.A[i] * np.power(T, m.B[i]) * np.exp(-m.EaR[i] / T)
        aij_X_sum = _seqsum(aij * X)
        aij_X_sum = m.is_third_body[i] * aij_X_sum + (1 - m.is_third_body[i])
        kf = kf_i * np.exp(_seqsum(vf_i * log_X))
        kb = kf_i / (np.exp(_seqsum((vb_i - vf_i) * g))
                     * ((101325 / m.nondim.P0 / T) ** m.vsum[i])) \
            * np.exp(_seqsum(vb_i * log_X))
        kf_l.append(kf)
        kb_l.append(kb)
        M_l.append(aij_X_sum)
    w = []
    J = np.empty((nr, nr) + T.shape[1:])
    for k in range(nr):
        Mk = m.species_M[k]
        terms = [(m.vb[i, k] - m.vf[i, k]) * M_l[i] * (kf_l[i] - kb_l[i]) for i in range(nreac)]
        w.append(Mk * _seqsum(np.stack(terms))[0, 0])
        for n in range(nr):
            Mn = m.species_M[n]
            Xn = Xc[n][None]
            tn = []
            for i in range(nreac):
                dv = m.vb[i, k] - m.vf[i, k]
                ain = m.third_body[i, n]
                tn.append(dv * (kf_l[i] - kb_l[i]) * (ain / Mn)
                          + 1 / (Mn * Xn) * dv * M_l[i] * (m.vf[i, n] * kf_l[i] - m.vb[i, n] * kb_l[i]))
            J[k, n] = Mk * _seqsum(np.stack(tn))[0, 0]
    S = np.moveaxis(np.stack(w), 0, -1)[..., None]               # (..., nr, 1)
    DSDU = np.moveaxis(np.moveaxis(J, 0, -1), 0, -1)             # (..., nr, nr)
    Amat = np.eye(nr) / dt - DSDU
    x = np.linalg.solve(Amat, S)
    return np.moveaxis(x[..., 0], -1, 0)


def reaction_source_terms(m, U, aux, dt):
    """reaction_model.py:183-193 (detailed_reaction)"""
    nY = nY_of(U)
    nd = U.ndim - 1
    rho = U[0:1]
    Y = fill_Y(U[nY:] / rho)
    rhoY = rho * Y
    T = aux[1:2]
    X = rhoY / _ex(m.species_M, nd)
    drhoY = construct_matrix_equation(m, T, X, dt)
    dY = drhoY / rho
    dY = np.clip(dY, -Y[0:-1], 1 - Y[0:-1])
    return np.concatenate([np.zeros_like(U[:nY]), rho * dY], axis=0)


# --------------------------------------------------------------------------
# boundaries  (boundary/*.py and the RDC notebook injector)
# --------------------------------------------------------------------------
def _pressure_outlet_state(m, state, gamma, T, normal_vel, Pb):
    """boundary_conditions_{1D,2D}/pressure_outlet.py:5-22"""
    nY = nY_of(state) if state.ndim > 2 else 3
    two_d = state.ndim == 3
    rho = state[0:1]
    u = state[1:2] / rho
    v = state[2:3] / rho if two_d else None
    Y = state[nY:] / rho
    R = get_R(m, Y)
    p = rho * (R * T)
    a = np.sqrt(gamma * p / rho)
    mask = normal_vel / a < 1
    rho_c = np.where(mask, Pb / (p / rho), rho)
    p_c = np.where(mask, Pb * np.ones_like(p), p)
    T_c = np.where(mask, p_c / (rho_c * R), T)
    _, gamma_c, h_c, _, _ = get_thermo(m, T_c, Y)
    if two_d:
        Ub = np.concatenate([rho_c, rho_c * u, rho_c * v,
                             rho_c * h_c - p_c + 0.5 * rho_c * (u ** 2 + v ** 2), rho_c * Y], axis=0)
    else:
        Ub = np.concatenate([rho_c, rho_c * u, rho_c * h_c - p_c + 0.5 * rho_c * (u ** 2), rho_c * Y], axis=0)
    return Ub, np.concatenate([gamma_c, T_c], axis=0)


def inj_model(m, p, Y_inj):
    """Injector pressure-feedback model of examples/janc_basic_example2.ipynb
    (``inj_model``, after Fievisohn et al. 2017): 20 bisection steps on the
    throat Mach number, nondimensional with manifold P0, T0."""
    A1, A3 = 1, 5
    A2 = A3 - A1
    R = get_R(m, Y_inj)
    gamma = 1.29
    C0 = np.sqrt(gamma * R * 1.0)
    P3 = p
    M1 = np.zeros_like(p)
    M2 = np.ones_like(p)
    for _ in range(20):
        M = 0.5 * (M1 + M2)
        P1 = 1.0 * (1 + (gamma - 1) / 2 * M ** 2) ** (-gamma / (gamma - 1))
        V1 = M * (1 + (gamma - 1) / 2 * M ** 2) ** (-0.5) * C0
        MFC = A1 * 1.0 / np.sqrt(1.0) * np.sqrt(gamma / R) * M * (1 + (gamma - 1) / 2 * M ** 2) ** (-(gamma + 1) / 2 / (gamma - 1))
        A = 0.5
        B = gamma / (gamma - 1) * P3 * A3 / MFC
        C = -gamma / (gamma - 1) * R * 1.0
        V3 = (-B + np.sqrt(B ** 2 - 4 * A * C)) / (2 * A)
        P2 = (MFC * (V3 - V1) - P1 * A1 + P3 * A3) / A2
        M2 = np.where(P2 >= P1, M, M2)
        M1 = np.where(P2 < P1, M, M1)
    rho_c = MFC / V3 / A3
    v_c = V3
    T_c = p / (R * rho_c)
    _, gamma_c, h_c, _, _ = get_thermo(m, T_c, Y_inj)
    return v_c, T_c, h_c, gamma_c


def _injector_state(m, state, aux, Yinj):
    """``bottom_boundary`` of examples/janc_basic_example2.ipynb on the first
    interior row; Yinj broadcasts as (8, nx, 1)."""
    rho, u, v, Y, p, a = U_to_prim(m, state, aux)
    T = aux[1:2]
    gamma = aux[0:1]
    _, _, h, R, _ = get_thermo(m, T, Y)
    u_inj = np.zeros_like(u)
    v_inj, T_inj, h_inj, g_inj = inj_model(m, p, Yinj)
    R_inj = get_R(m, Yinj)
    rho_inj = p / (R_inj * T_inj)
    blk = p >= 1.0
    rho_c = np.where(blk, rho, rho_inj)
    u_c = np.where(blk, u, u_inj)
    v_c = np.where(blk, -v, v_inj)
    T_c = np.where(blk, T, T_inj)
    p_c = p
    h_c = np.where(blk, h, h_inj)
    Y_c = np.where(np.tile(blk, (Yinj.shape[0], 1, 1)), Y, Yinj)
    g_c = np.where(blk, gamma, g_inj)
    Ub = np.concatenate([rho_c, rho_c * u_c, rho_c * v_c,
                         rho_c * h_c - p_c + 0.5 * rho_c * (u_c ** 2 + v_c ** 2), rho_c * Y_c], axis=0)
    return Ub, np.concatenate([g_c, T_c], axis=0)


def _bc_side(m, kind, side, Ub, auxb, theta):
    """One side's 3 ghost layers from the 3 boundary-adjacent layers
    (boundary_conditions_{1D,2D}/*.py).  ``side`` in L/R/B/T; layers are
    along axis 1 (L/R) or axis 2 (B/T), ordered as in the padded array."""
    if callable(kind):  # a user function of the 3 adjacent layers (boundary.py:16-21, 37-42)
        return kind(Ub, auxb, theta)
    ax = 1 if side in "LR" else 2
    lo = side in "LB"
    two_d = Ub.ndim == 3

    def take(a, j):
        return np.take(a, [j], axis=ax)

    def cat(parts):
        return np.concatenate(parts, axis=ax)

    if kind == "zero_gradient" or kind == "no_slip_wall":
        order = [2, 1, 0] if lo else [-1, -2, -3]
        U = cat([take(Ub, j) for j in order])
        A = cat([take(auxb, j) for j in order])
        if kind == "no_slip_wall":
            U = U.copy()
            if two_d:
                U[1:3] *= -1
            else:
                U[1:2] *= -1
        return U, A
    if kind == "slip_wall":
        j = 0 if lo else -1
        U = cat([take(Ub, j)] * 3).copy()
        A = cat([take(auxb, j)] * 3)
        mom = 1 if (side in "LR") else 2
        U[mom:mom + 1] *= -1
        return U, A
    if kind == "pressure_outlet":
        j = 0 if lo else -1
        st, ga, Tt = take(Ub, j), take(auxb[0:1], j), take(auxb[1:2], j)
        mom = 1 if side in "LR" else 2
        nv = st[mom:mom + 1] / st[0:1]
        if lo:
            nv = -nv
        Us, As = _pressure_outlet_state(m, st, ga, Tt, nv, theta["Pb"])
        return cat([Us] * 3), cat([As] * 3)
    if kind == "rdc_injector":
        assert side == "B" and two_d
        st, au = Ub[:, :, 0:1], auxb[:, :, 0:1]
        Yinj = np.asarray(theta["Yinj"])
        if Yinj.ndim == 1:
            Yinj = np.tile(Yinj[:, None, None], (1, Ub.shape[1], 1))
        Us, As = _injector_state(m, st, au, Yinj)
        return np.tile(Us, (1, 1, 3)), np.tile(As, (1, 1, 3))
    raise KeyError(kind)


def boundary_conditions(m, U, aux, bc, theta=None):
    """Periodic pad (boundary_padding.py:4-25, node-periodic quirk), then
    overwrite L, R (, B, T) in that order (boundary.py:120-132)."""
    f = np.concatenate([U, aux], axis=0)
    f = np.concatenate([f[:, -4:-3], f[:, -3:-2], f[:, -2:-1], f, f[:, 1:2], f[:, 2:3], f[:, 3:4]], axis=1)
    two_d = U.ndim == 3
    if two_d:
        f = np.concatenate([f[:, :, -4:-3], f[:, :, -3:-2], f[:, :, -2:-1], f,
                            f[:, :, 1:2], f[:, :, 2:3], f[:, :, 3:4]], axis=2)
    Up, Ap = f[:-2].copy(), f[-2:].copy()
    sides = (("L", "left_boundary"), ("R", "right_boundary"))
    if two_d:
        sides += (("B", "bottom_boundary"), ("T", "top_boundary"))
    return _apply_sides(m, Up, Ap, bc, theta, sides)


def parallel_boundary_conditions(m, Us, auxs, r, bc, theta=None):
    """Slab r of the reference's parallel mode (parallel/boundary.py:6-25 with
    parallel/boundary_padding.py:6-27): the x pad is a ring exchange of 3
    columns with the neighbouring slabs (exchange_halo, cell-periodic across
    the domain's ends), the y pad the node-periodic one; then the left
    condition on slab 0 only, the right on the last slab only, bottom and top
    on every slab."""
    P = len(Us)
    f = [np.concatenate([U, a], axis=0) for U, a in zip(Us, auxs)]
    fx = np.concatenate([f[(r - 1) % P][:, -3:], f[r], f[(r + 1) % P][:, :3]], axis=1)
    two_d = Us[r].ndim == 3
    if two_d:
        fx = np.concatenate([fx[:, :, -4:-3], fx[:, :, -3:-2], fx[:, :, -2:-1], fx,
                             fx[:, :, 1:2], fx[:, :, 2:3], fx[:, :, 3:4]], axis=2)
    Up, Ap = fx[:-2].copy(), fx[-2:].copy()
    sides = ()
    if r == 0:
        sides += (("L", "left_boundary"),)
    if r == P - 1:
        sides += (("R", "right_boundary"),)
    if two_d:
        sides += (("B", "bottom_boundary"), ("T", "top_boundary"))
    return _apply_sides(m, Up, Ap, bc, theta, sides)


def _apply_sides(m, Up, Ap, bc, theta, sides):
    two_d = Up.ndim == 3
    for s, key in sides:
        kind = bc[key]
        if kind == "periodic":
            continue
        if two_d:
            sl = {"L": (slice(None), slice(3, 6), slice(3, -3)), "R": (slice(None), slice(-6, -3), slice(3, -3)),
                  "B": (slice(None), slice(3, -3), slice(3, 6)), "T": (slice(None), slice(3, -3), slice(-6, -3))}[s]
            dst = {"L": (slice(None), slice(0, 3), slice(3, -3)), "R": (slice(None), slice(-3, None), slice(3, -3)),
                   "B": (slice(None), slice(3, -3), slice(0, 3)), "T": (slice(None), slice(3, -3), slice(-3, None))}[s]
        else:
            sl = {"L": (slice(None), slice(3, 6)), "R": (slice(None), slice(-6, -3))}[s]
            dst = {"L": (slice(None), slice(0, 3)), "R": (slice(None), slice(-3, None))}[s]
        Ug, Ag = _bc_side(m, kind, s, Up[sl], Ap[sl], theta)
        Up[dst] = Ug
        Ap[dst] = Ag
    return Up, Ap


# --------------------------------------------------------------------------
# LF splitting + WENO5-JS  (flux_splitting/LF.py, reconstruction/WENO5_JS.py)
# --------------------------------------------------------------------------
_EPS, _C1, _C2, _C3 = 1e-6, 1 / 10, 3 / 5, 3 / 10


def _sq(x):
    """jnp.power(x, 2) with an integer exponent is x*x (lax.integer_pow)."""
    return x * x


def _weno_L(fjm2, fjm1, fj, fjp1, fjp2):
    IS1 = 1 / 4 * _sq(fjm2 - 4 * fjm1 + 3 * fj) + 13 / 12 * _sq(fjm2 - 2 * fjm1 + fj)
    IS2 = 1 / 4 * _sq(fjm1 - fjp1) + 13 / 12 * _sq(fjm1 - 2 * fj + fjp1)
    IS3 = 1 / 4 * _sq(3 * fj - 4 * fjp1 + fjp2) + 13 / 12 * _sq(fj - 2 * fjp1 + fjp2)
    a1 = _C1 / _sq(_EPS + IS1)
    a2 = _C2 / _sq(_EPS + IS2)
    a3 = _C3 / _sq(_EPS + IS3)
    w1 = a1 / (a1 + a2 + a3)
    w2 = a2 / (a1 + a2 + a3)
    w3 = a3 / (a1 + a2 + a3)
    q1 = 1 / 3 * fjm2 - 7 / 6 * fjm1 + 11 / 6 * fj
    q2 = -1 / 6 * fjm1 + 5 / 6 * fj + 1 / 3 * fjp1
    q3 = 1 / 3 * fj + 5 / 6 * fjp1 - 1 / 6 * fjp2
    return w1 * q1 + w2 * q2 + w3 * q3


def _weno_R(fjm2, fjm1, fj, fjp1, fjp2):
    IS1 = 1 / 4 * _sq(fjp2 - 4 * fjp1 + 3 * fj) + 13 / 12 * _sq(fjp2 - 2 * fjp1 + fj)
    IS2 = 1 / 4 * _sq(fjp1 - fjm1) + 13 / 12 * _sq(fjp1 - 2 * fj + fjm1)
    IS3 = 1 / 4 * _sq(3 * fj - 4 * fjm1 + fjm2) + 13 / 12 * _sq(fj - 2 * fjm1 + fjm2)
    a1 = _C1 / _sq(_EPS + IS1)
    a2 = _C2 / _sq(_EPS + IS2)
    a3 = _C3 / _sq(_EPS + IS3)
    w1 = a1 / (a1 + a2 + a3)
    w2 = a2 / (a1 + a2 + a3)
    w3 = a3 / (a1 + a2 + a3)
    q1 = 1 / 3 * fjp2 - 7 / 6 * fjp1 + 11 / 6 * fj
    q2 = -1 / 6 * fjp1 + 5 / 6 * fj + 1 / 3 * fjm1
    q3 = 1 / 3 * fj + 5 / 6 * fjm1 - 1 / 6 * fjm2
    return w1 * q1 + w2 * q2 + w3 * q3


def _interface_L(q, axis, other_interior):
    """WENO5_JS.interface_L_{x,y}: face values from cells j-2..j+2."""
    def s(a, b):
        idx = [slice(None)] * q.ndim
        idx[axis] = slice(a, b)
        if other_interior is not None:
            idx[other_interior] = slice(3, -3)
        return q[tuple(idx)]
    return _weno_L(s(0, -5), s(1, -4), s(2, -3), s(3, -2), s(4, -1))


def _interface_R(q, axis, other_interior):
    def s(a, b):
        idx = [slice(None)] * q.ndim
        idx[axis] = slice(a, b)
        if other_interior is not None:
            idx[other_interior] = slice(3, -3)
        return q[tuple(idx)]
    return _weno_R(s(1, -4), s(2, -3), s(3, -2), s(4, -1), s(5, None))


def _minmod(x, y):
    """min_mod_limiter (reconstruction/MUSCL.py:4-7)"""
    mask1 = np.minimum(x * np.sign(y), y * np.sign(x))
    mask = np.maximum(np.zeros_like(mask1), mask1)
    return np.sign(x) * mask


def _muscl(q, axis, other_interior, left, k=1 / 3, beta=1.0):
    """MUSCL interface_L / interface_R (reconstruction/MUSCL.py, 1D and 2D):
    face states of cells 1 .. n+4 of the padded axis, minmod-limited."""
    def s(a, b):
        idx = [slice(None)] * q.ndim
        idx[axis] = slice(a, b)
        if other_interior is not None:
            idx[other_interior] = slice(3, -3)
        return q[tuple(idx)]

    def t(U, a, b):
        idx = [slice(None)] * U.ndim
        idx[axis] = slice(a, b)
        return U[tuple(idx)]
    U = s(1, -1)
    d_minus = t(U, 1, -1) - t(U, None, -2)
    d_plus = t(U, 2, None) - t(U, 1, -1)
    phi_fw = _minmod(d_plus, beta * d_minus)
    phi_bw = _minmod(d_minus, beta * d_plus)
    if left:
        s_L = 1 / 4 * ((1 - k) * phi_bw + (1 + k) * phi_fw)
        return t(U, 1, -2) + t(s_L, None, -1)
    s_R = 1 / 4 * ((1 - k) * phi_fw + (1 + k) * phi_bw)
    return t(U, 2, -1) - t(s_R, 1, None)


def _recon(q, axis, other_interior, left, recon):
    if recon == "MUSCL":
        return _muscl(q, axis, other_interior, left)
    return (_interface_L if left else _interface_R)(q, axis, other_interior)


def split_flux_1d(m, U, aux):
    """solver_1D/flux_splitting/LF.py:4-13"""
    rho, u, Y, p, a = U_to_prim(m, U, aux)
    rhoE = U[2:3]
    zx = 1.0
    F = zx * np.concatenate([rho * u, rho * u ** 2 + p, u * (rhoE + p), rho * u * Y], axis=0)
    um = zx * np.nanmax(abs(u) + a)
    return 0.5 * (F + um * U), 0.5 * (F - um * U)


def split_flux_2d(m, ixy, U, aux):
    """solver_2D/flux_splitting/LF.py:4-16"""
    rho, u, v, Y, p, a = U_to_prim(m, U, aux)
    rhoE = U[3:4]
    zx = (ixy == 1) * 1.0
    zy = (ixy == 2) * 1.0
    F = zx * np.concatenate([rho * u, rho * u ** 2 + p, rho * u * v, u * (rhoE + p), rho * u * Y], axis=0) \
        + zy * np.concatenate([rho * v, rho * u * v, rho * v ** 2 + p, v * (rhoE + p), rho * v * Y], axis=0)
    um = np.nanmax(abs(u) + a)
    vm = np.nanmax(abs(v) + a)
    th = zx * um + zy * vm
    return 0.5 * (F + th * U), 0.5 * (F - th * U)


def _sw_combine(theta, a, H1, H2, H4):
    """Eigenvalue groups of flux_splitting/SW.py (smoothed |lambda|)."""
    lambda1, lambda2, lambda4 = theta - a, theta, theta + a
    eps = 1e-6
    lap1 = 0.5 * (lambda1 + np.sqrt(np.power(lambda1, 2) + eps ** 2))
    lam1 = 0.5 * (lambda1 - np.sqrt(np.power(lambda1, 2) + eps ** 2))
    lap2 = 0.5 * (lambda2 + np.sqrt(np.power(lambda2, 2) + eps ** 2))
    lam2 = 0.5 * (lambda2 - np.sqrt(np.power(lambda2, 2) + eps ** 2))
    lap4 = 0.5 * (lambda4 + np.sqrt(np.power(lambda4, 2) + eps ** 2))
    lam4 = 0.5 * (lambda4 - np.sqrt(np.power(lambda4, 2) + eps ** 2))
    return lap1 * H1 + lap2 * H2 + lap4 * H4, lam1 * H1 + lam2 * H2 + lam4 * H4


def split_sw_2d(m, ixy, U, aux):
    """solver_2D/flux_splitting/SW.py:4-37 (Steger-Warming)"""
    rho, u, v, Y, p, a = U_to_prim(m, U, aux)
    rhoE = U[3:4]
    gamma = aux[0:1]
    zx = (ixy == 1) * 1.0
    zy = (ixy == 2) * 1.0
    theta = zx * u + zy * v
    H1 = (1 / (2 * gamma)) * np.concatenate([rho, rho * u - rho * a * zx, rho * v - rho * a * zy,
                                             rhoE + p - rho * a * theta, rho * Y], axis=0)
    H2 = ((gamma - 1) / gamma) * np.concatenate([rho, rho * u, rho * v, 0.5 * rho * (u ** 2 + v ** 2), rho * Y],
                                                axis=0)
    H4 = (1 / (2 * gamma)) * np.concatenate([rho, rho * u + rho * a * zx, rho * v + rho * a * zy,
                                             rhoE + p + rho * a * theta, rho * Y], axis=0)
    return _sw_combine(theta, a, H1, H2, H4)


def split_sw_1d(m, U, aux):
    """solver_1D/flux_splitting/SW.py:4-36 with J = 1 and zx = 1 (the
    reference's 1D flux_splitting calls split_flux(U, aux) without the
    `metrics` argument this function declares, so the 1D SW path raises a
    TypeError there; this is the arithmetic the function states)."""
    rho, u, Y, p, a = U_to_prim(m, U, aux)
    rhoE = U[2:3]
    gamma = aux[0:1]
    J, zx = 1.0, 1.0
    theta = zx * u
    H1 = J * (1 / (2 * gamma)) * np.concatenate([rho, rho * u - rho * a * zx, rhoE + p - rho * a * theta,
                                                 rho * Y], axis=0)
    H2 = J * ((gamma - 1) / gamma) * np.concatenate([rho, rho * u, 0.5 * rho * (u ** 2), rho * Y], axis=0)
    H4 = J * (1 / (2 * gamma)) * np.concatenate([rho, rho * u + rho * a * zx, rhoE + p + rho * a * theta,
                                                 rho * Y], axis=0)
    return _sw_combine(theta, a, H1, H2, H4)


def total_flux(m, Up, Ap, dx, dy=None, recon="WENO5_JS", split="LF"):
    """flux_splitting (solver_1D/flux.py:51-58, solver_2D/flux.py:56-68) on
    the ghost-padded arrays; returns -(dF/dx [+ dG/dy])."""
    if Up.ndim == 2:
        Fplus, Fminus = (split_sw_1d if split == "SW" else split_flux_1d)(m, Up, Ap)
        F = _recon(Fplus, 1, None, True, recon) + _recon(Fminus, 1, None, False, recon)
        dF = F[:, 1:] - F[:, :-1]
        return -(dF / dx)
    sf = split_sw_2d if split == "SW" else split_flux_2d
    Fplus, Fminus = sf(m, 1, Up, Ap)
    Gplus, Gminus = sf(m, 2, Up, Ap)
    F = _recon(Fplus, 1, 2, True, recon) + _recon(Fminus, 1, 2, False, recon)
    G = _recon(Gplus, 2, 1, True, recon) + _recon(Gminus, 2, 1, False, recon)
    dF = F[:, 1:, :] - F[:, :-1, :]
    dG = G[:, :, 1:] - G[:, :, :-1]
    return -(dF / dx + dG / dy)


# --------------------------------------------------------------------------
# Godunov path: WENO5-JS on primitives + HLLC / AUSMPW+
# (solver_{1D,2D}/flux.py godunov_flux, riemann_solver/HLLC.py,
#  riemann_solver/AUSMPW_plus.py)
# --------------------------------------------------------------------------
def _face_thermo(m, rho, p, Y):
    """T = p / (R rho) of a reconstructed face state, then its gamma and h
    (HLLC.py:8-12 in 2D, :7-11 in 1D; AUSMPW_plus.py:86-92 / 62-66)."""
    R = get_R(m, Y)
    T = p / (R * rho)
    _, gamma, h, _, _ = get_thermo(m, T, Y)
    return gamma, h


def _hllc(m, qL, qR, dim, n):
    """HLLC flux through faces with normal velocity component n (1: x,
    2: y) of primitive face states q = [rho, u, (v), p, Y]
    (solver_2D/riemann_solver/HLLC.py:15-43 x, :45-73 y; solver_1D HLLC.py:13-42)."""
    ip = 1 + dim
    rho_L, rho_R = qL[0:1], qR[0:1]
    p_L, p_R = qL[ip:ip + 1], qR[ip:ip + 1]
    Y_L, Y_R = qL[ip + 1:], qR[ip + 1:]
    gamma_L, h_L = _face_thermo(m, rho_L, p_L, Y_L)
    gamma_R, h_R = _face_thermo(m, rho_R, p_R, Y_R)
    a_L = np.sqrt(gamma_L * p_L / rho_L)
    a_R = np.sqrt(gamma_R * p_R / rho_R)
    vel_L = [qL[1 + k:2 + k] for k in range(dim)]
    vel_R = [qR[1 + k:2 + k] for k in range(dim)]
    un_L, un_R = vel_L[n - 1], vel_R[n - 1]
    if dim == 2:
        E_L = rho_L * h_L - p_L + 0.5 * rho_L * (vel_L[0] ** 2 + vel_L[1] ** 2)
        E_R = rho_R * h_R - p_R + 0.5 * rho_R * (vel_R[0] ** 2 + vel_R[1] ** 2)
    else:
        E_L = rho_L * h_L - p_L + 0.5 * rho_L * (vel_L[0] ** 2)
        E_R = rho_R * h_R - p_R + 0.5 * rho_R * (vel_R[0] ** 2)
    s_L = np.minimum(un_L - a_L, un_R - a_R)
    s_R = np.maximum(un_L + a_L, un_R + a_R)
    s_M = (p_R - p_L + rho_L * un_L * (s_L - un_L) - rho_R * un_R * (s_R - un_R)) / \
        (rho_L * (s_L - un_L) - rho_R * (s_R - un_R))

    def side(rho, vel, un, p, E, Y, s):
        U = np.concatenate([rho] + [rho * v for v in vel] + [E, rho * Y], axis=0)
        star_vel = [s_M if k == n - 1 else vel[k] for k in range(dim)]
        U_M = rho * (s - un) / (s - s_M) * np.concatenate(
            [np.ones_like(s_M)] + star_vel + [E / rho + (s_M - un) * (s_M + p / (rho * (s - un))), Y], axis=0)
        mom = []
        for k in range(dim):
            if k == n - 1:
                mom.append(rho * un ** 2 + p)
            elif n == 1:
                mom.append(rho * un * vel[k])      # rho u v through x faces
            else:
                mom.append(rho * vel[k] * un)      # rho u v through y faces
        F = np.concatenate([rho * un] + mom + [un * (E + p), rho * un * Y], axis=0)
        return F, F + s * (U_M - U)

    F_L, F_L_M = side(rho_L, vel_L, un_L, p_L, E_L, Y_L, s_L)
    F_R, F_R_M = side(rho_R, vel_R, un_R, p_R, E_R, Y_R, s_R)
    cond1 = s_L >= 0
    cond2 = np.logical_and(s_L <= 0, s_M >= 0)
    cond3 = np.logical_and(s_M <= 0, s_R >= 0)
    F1 = np.where(cond1, F_L, F_R)
    F2 = np.where(cond2, F_L_M, F1)
    return np.where(cond3, F_R_M, F2)


def _split_M_and_P(M):
    """AUSMPW_plus.py:5-11"""
    ind = np.abs(M) <= 1
    Mplus = np.where(ind, 1 / 4 * (M + 1) ** 2, 1 / 2 * (M + np.abs(M)))
    Mminus = np.where(ind, -1 / 4 * (M - 1) ** 2, 1 / 2 * (M - np.abs(M)))
    Pplus = np.where(ind, 1 / 4 * (M + 1) ** 2 * (2 - M), 1 / 2 * (1 + np.sign(M)))
    Pminus = np.where(ind, 1 / 4 * (M - 1) ** 2 * (2 + M), 1 / 2 * (1 - np.sign(M)))
    return Mplus, Mminus, Pplus, Pminus


def _ausmpw(m, qL, qR, dim, n):
    """AUSMPW+ flux (solver_2D/riemann_solver/AUSMPW_plus.py:13-24, 77-131;
    solver_1D AUSMPW_plus.py).  At y faces the reference takes gamma_R from
    the x-face states (2D AUSMPW_plus.py:54), whose shape does not broadcast
    with the y-face arrays, so the reference's 2D AUSMPW+ cannot run; the
    y faces here use their own gamma_R."""
    ip = 1 + dim
    rho_L, rho_R = qL[0:1], qR[0:1]
    p_L, p_R = qL[ip:ip + 1], qR[ip:ip + 1]
    Y_L, Y_R = qL[ip + 1:], qR[ip + 1:]
    gamma_L, h_L = _face_thermo(m, rho_L, p_L, Y_L)
    gamma_R, h_R = _face_thermo(m, rho_R, p_R, Y_R)
    un_L, un_R = qL[n:n + 1], qR[n:n + 1]
    c_L = np.sqrt(gamma_L * p_L / rho_L)
    c_R = np.sqrt(gamma_R * p_R / rho_R)
    c = 0.5 * (c_L + c_R)
    M_L, M_R = un_L / c, un_R / c

    def phi(rho, q, h, Y):
        vel = [q[1 + k:2 + k] for k in range(dim)]
        kin = vel[0] ** 2 + vel[1] ** 2 if dim == 2 else vel[0] ** 2
        return np.concatenate([rho] + [rho * v for v in vel] + [rho * h + 0.5 * rho * kin, rho * Y], axis=0)

    phi_L, phi_R = phi(rho_L, qL, h_L, Y_L), phi(rho_R, qR, h_R, Y_R)
    M_L_plus, _, P_L_plus, _ = _split_M_and_P(M_L)
    _, M_R_minus, _, P_R_minus = _split_M_and_P(M_R)
    p_s = P_L_plus * p_L + P_R_minus * p_R
    mask = np.minimum(p_L / p_R, p_R / p_L)
    w = 1 - mask * (mask * mask)  # jnp x**3 is lax.integer_pow: x * (x * x)
    fL = np.where(np.abs(M_L) < 1.0, p_L / p_s - 1, np.zeros_like(p_L))
    fR = np.where(np.abs(M_R) < 1.0, p_R / p_s - 1, np.zeros_like(p_R))
    ind = M_L_plus + M_R_minus >= 0
    M_L_av = np.where(ind, M_L_plus + M_R_minus * ((1 - w) * (1 + fR) - fL), M_L_plus * w * (1 + fL))
    M_R_av = np.where(ind, M_R_minus * w * (1 + fR), M_R_minus + M_L_plus * ((1 - w) * (1 + fL) - fR))
    P_L = np.zeros_like(phi_L)
    P_L[n:n + 1] = p_L
    P_R = np.zeros_like(phi_R)
    P_R[n:n + 1] = p_R
    return M_L_av * c * phi_L + M_R_av * c * phi_R + (P_L_plus * P_L + P_R_minus * P_R)


RIEMANN = {"HLLC": _hllc, "AUSMPW_plus": _ausmpw}


def godunov_flux(m, Up, Ap, dx, dy=None, riemann="HLLC", recon="WENO5_JS"):
    """godunov_flux (solver_1D/flux.py:41-49, solver_2D/flux.py:43-54) on the
    ghost-padded arrays: primitives q = [rho, u, (v), p, Y], WENO5-JS
    left / right face states per component, the Riemann flux, and
    -(dF/dx [+ dG/dy])."""
    rs = RIEMANN[riemann]
    if Up.ndim == 2:
        rho, u, Y, p, a = U_to_prim(m, Up, Ap)
        q = np.concatenate([rho, u, p, Y], axis=0)
        F = rs(m, _recon(q, 1, None, True, recon), _recon(q, 1, None, False, recon), 1, 1)
        dF = F[:, 1:] - F[:, :-1]
        return -(dF / dx)
    rho, u, v, Y, p, a = U_to_prim(m, Up, Ap)
    q = np.concatenate([rho, u, v, p, Y], axis=0)
    F = rs(m, _recon(q, 1, 2, True, recon), _recon(q, 1, 2, False, recon), 2, 1)
    G = rs(m, _recon(q, 2, 1, True, recon), _recon(q, 2, 1, False, recon), 2, 2)
    dF = F[:, 1:, :] - F[:, :-1, :]
    dG = G[:, :, 1:] - G[:, :, :-1]
    return -(dF / dx + dG / dy)


# --------------------------------------------------------------------------
# viscous flux, laminar (solver_{1D,2D}/flux.py viscous_flux_node /
# viscous_flux, model/transport_model.py, finite_difference/CENTRAL6.py,
# reconstruction/CENTRAL6.py)
# --------------------------------------------------------------------------
class Transport:
    """set_transport (transport_model.py:26-104) for the laminar model."""

    def __init__(self, cfg):
        self.mu_ref, self.T_ref, self.S, self.nu0 = 1.716e-5, 273.15, 110.4, 1e-4
        self.Pr, self.Pr_t, self.Sc, self.Sc_t, self.Le, self.Le_t = 0.72, 0.72, 0.72, 0.72, 1.0, 1.0
        self.k0, self.D0 = 0.0, 0.0
        self.nu_type, self.k_type, self.D_type = "Sutherland", "Prandtl number", "Lewis number"
        if cfg["viscosity_model"] == "constant":
            self.nu_type = "constant"
            self.nu0 = cfg["dynamic_viscosity"]
        elif cfg["viscosity_model"] == "Sutherland":
            self.mu_ref = cfg.get("reference_viscosity", self.mu_ref)
            self.T_ref = cfg.get("reference_temperature", self.T_ref)
            self.S = cfg.get("effective_temperature", self.S)
        else:
            raise KeyError("Only 'Sutherland' and 'constant' viscosity model are supported.")
        if cfg["thermal_conductivity_model"] == "constant":
            self.k_type = "constant"
            self.k0 = cfg["thermal_conductivity"]
        elif cfg["thermal_conductivity_model"] == "Prandtl number":
            self.Pr = cfg["Pr"]
        else:
            raise KeyError("Only 'Prandtl number' and 'constant' thermal conductivity model are supported.")
        if cfg["species_diffusivity_model"] == "constant":
            self.D_type = "constant"
            self.D0 = cfg["species_diffusivity"]
        elif cfg["species_diffusivity_model"] == "Schmidt number":
            self.Sc = cfg["Sc"]
            self.Le = self.Sc / self.Pr
        elif cfg["species_diffusivity_model"] == "Lewis number":
            self.Le = cfg["Le"]
            self.Sc = self.Le * self.Pr
        else:
            raise KeyError("Only 'Schmidt number', 'Lewis number', and 'constant' species diffusivity "
                           "model are supported.")
        self.model, self.LES_model = "laminar", None
        if "turbulence_model" in cfg:
            if cfg["turbulence_model"] == "LES":
                self.model = "LES"
                assert "LES_model" in cfg, "Please specify the SGS model of LES."
                self.LES_model = cfg["LES_model"]
                assert "Pr_t" in cfg
                assert ("Le_t" in cfg) or ("Sc_t" in cfg)
                self.Pr_t = cfg["Pr_t"]
                if "Le_t" in cfg:
                    self.Le_t = cfg["Le_t"]
                    self.Sc_t = self.Le_t * self.Pr_t
                else:
                    self.Sc_t = cfg["Sc_t"]
                    self.Le_t = self.Sc_t / self.Pr_t
            elif cfg["turbulence_model"] != "laminar":
                raise KeyError("Only 'laminar' and 'LES' model are supported.")

    def mu(self, rho, T):
        """mu_Sutherland / mu_constant (:106-112), the laminar part"""
        if self.nu_type == "Sutherland":
            return self.mu_ref * (T / self.T_ref) ** 1.5 * (self.T_ref + self.S) / (T + self.S)
        return rho * self.nu0

    def mu_total(self, rho, T, dx, dy, du_dx, du_dy, dv_dx, dv_dy):
        """transport_model.mu (:117-130): (mu, mu_t), mu = laminar + mu_t for
        LES with the 2D Vreman model (model/LES/Verman.py:5-27, c = 0.07)."""
        mu = self.mu(rho, T)
        if self.model != "LES":
            return mu, 0.0
        if self.LES_model != "Verman" or dy is None:
            raise KeyError(f"{self.LES_model}_{'2D' if dy is not None else '1D'}")
        d1, d2 = dx, dy
        a11, a12 = du_dx, dv_dx
        a21, a22 = du_dy, dv_dy
        b11_x, b12_x = (d1 ** 2) * a11 * a11, (d1 ** 2) * a11 * a12
        b22_x = (d1 ** 2) * a12 * a12
        b11_y, b12_y = (d2 ** 2) * a21 * a21, (d2 ** 2) * a21 * a22
        b22_y = (d2 ** 2) * a22 * a22
        b11, b12, b22 = b11_x + b11_y, b12_x + b12_y, b22_x + b22_y
        B_b = np.abs(b11 * b22 - b12 ** 2)
        B_b = np.where(B_b >= 0.0, B_b, np.zeros_like(B_b))
        a_sum = a11 ** 2 + a12 ** 2 + a21 ** 2 + a22 ** 2
        with np.errstate(divide="ignore", invalid="ignore"):
            ratio = np.where(a_sum > 0.0, B_b / a_sum, np.zeros_like(a_sum))
        mu_t = rho * 0.07 * np.sqrt(ratio)
        return mu + mu_t, mu_t

    def kappa(self, mu, cp, mu_t=0.0):
        """kappa_Pr / kappa_constant (:133-137)"""
        if self.k_type == "Prandtl number":
            return mu * cp / self.Pr + mu_t * cp / self.Pr_t
        return self.k0 + mu_t * cp / self.Pr_t

    def D(self, mu, rho, cp_i, mu_t=0.0):
        """D_Le / D_constant (:146-157)"""
        if self.D_type == "Lewis number" or self.D_type == "Schmidt number":
            k_i = (self.k_type == "Prandtl number") * mu * cp_i / self.Pr + (self.k_type == "constant") * self.k0
            rhoD_i = k_i / (self.Le * cp_i)
            k_t = mu_t / self.Pr_t
            rhoD_t = k_t / (self.Le_t * cp_i)
            return (rhoD_i + rhoD_t) / rho
        k_t = mu_t / self.Pr_t
        rhoD_t = k_t / self.Le_t * cp_i
        return self.D0 + rhoD_t / rho


def _d_axis(f, d, axis):
    """finite_difference/CENTRAL6.py d_dx / d_dy: sixth-order central inside,
    (4th, 2nd, 1st)-order one-sided forms at the first and last three."""
    def s(a, b):
        idx = [slice(None)] * f.ndim
        idx[axis] = slice(a, b)
        return f[tuple(idx)]
    n = f.shape[axis]
    center = (-s(0, n - 6) + 9 * s(1, n - 5) - 45 * s(2, n - 4) + 45 * s(4, n - 2) - 9 * s(5, n - 1)
              + s(6, n)) / (60 * d)
    left3 = (s(0, 1) - 8 * s(1, 2) + 8 * s(3, 4) - s(4, 5)) / (12 * d)
    left2 = (s(2, 3) - s(0, 1)) / (2 * d)
    left1 = (s(1, 2) - s(0, 1)) / d
    right1 = (s(n - 5, n - 4) - 8 * s(n - 4, n - 3) + 8 * s(n - 2, n - 1) - s(n - 1, n)) / (12 * d)
    right2 = (s(n - 1, n) - s(n - 3, n - 2)) / (2 * d)
    right3 = (s(n - 1, n) - s(n - 2, n - 1)) / d
    return np.concatenate([left1, left2, left3, center, right1, right2, right3], axis=axis)


def _central6_interface(fv, axis, other_interior):
    """reconstruction/CENTRAL6.py interface_x / interface_y"""
    def s(a, b):
        idx = [slice(None)] * fv.ndim
        idx[axis] = slice(a, b)
        if other_interior is not None:
            idx[other_interior] = slice(3, -3)
        return fv[tuple(idx)]
    return (3 * s(0, -5) - 25 * s(1, -4) + 150 * s(2, -3) + 150 * s(3, -2) - 25 * s(4, -1)
            + 3 * s(5, None)) / 256


def viscous_flux(m, tr, Up, Ap, dx, dy=None):
    """viscous_flux (solver_2D/flux.py:70-115, solver_1D/flux.py:67-99) on the
    ghost-padded arrays (corners keep the periodic wrap): returns
    dF_v/dx [+ dG_v/dy] (added to the advective -(dF/dx + dG/dy))."""
    T = Ap[1:2]
    cp_k, _, h_k = get_thermo_properties(m, T[0])
    if Up.ndim == 2:
        rho, u, Y, p, a = U_to_prim(m, Up, Ap)
        cp = get_thermo(m, T, Y)[0]
        Yf = fill_Y(Y)
        du_dx = _d_axis(u, dx, 1)
        dT_dx = _d_axis(T, dx, 1)
        dY_dx = _d_axis(Yf, dx, 1)
        mu, mu_t = tr.mu_total(rho, T, dx, None, du_dx, None, None, None)
        k = tr.kappa(mu, cp, mu_t)
        D_k = tr.D(mu, rho, cp_k, mu_t)
        div_u = du_dx
        tau_xx = 2 * mu * du_dx - 2 / 3 * mu * div_u
        qx = -k * dT_dx
        jx = -rho * D_k * dY_dx
        ex = _seqsum(jx * h_k)
        F_hat = np.concatenate([np.zeros_like(rho), tau_xx, u * tau_xx - qx - ex, -jx[0:-1]], axis=0)
        Fi = _central6_interface(F_hat, 1, None)
        return (Fi[:, 1:] - Fi[:, :-1]) / dx
    rho, u, v, Y, p, a = U_to_prim(m, Up, Ap)
    cp = get_thermo(m, T, Y)[0]
    Yf = fill_Y(Y)
    du_dx, du_dy = _d_axis(u, dx, 1), _d_axis(u, dy, 2)
    dv_dx, dv_dy = _d_axis(v, dx, 1), _d_axis(v, dy, 2)
    dT_dx, dT_dy = _d_axis(T, dx, 1), _d_axis(T, dy, 2)
    dY_dx, dY_dy = _d_axis(Yf, dx, 1), _d_axis(Yf, dy, 2)
    mu, mu_t = tr.mu_total(rho, T, dx, dy, du_dx, du_dy, dv_dx, dv_dy)
    k = tr.kappa(mu, cp, mu_t)
    D_k = tr.D(mu, rho, cp_k, mu_t)
    lam = -2 / 3 * mu
    S12 = 0.5 * (du_dy + dv_dx)
    div_u = du_dx + dv_dy
    tau_xx = 2 * mu * du_dx + lam * div_u
    tau_yy = 2 * mu * dv_dy + lam * div_u
    tau_xy = 2 * mu * S12
    qx, qy = -k * dT_dx, -k * dT_dy
    jx, jy = -rho * D_k * dY_dx, -rho * D_k * dY_dy
    ex, ey = _seqsum(jx * h_k), _seqsum(jy * h_k)
    F_hat = np.concatenate([np.zeros_like(rho), tau_xx, tau_xy, u * tau_xx + v * tau_xy - qx - ex, -jx[0:-1]], axis=0)
    G_hat = np.concatenate([np.zeros_like(rho), tau_xy, tau_yy, u * tau_xy + v * tau_yy - qy - ey, -jy[0:-1]], axis=0)
    Fi = _central6_interface(F_hat, 1, 2)
    Gi = _central6_interface(G_hat, 2, 1)
    return (Fi[:, 1:, :] - Fi[:, :-1, :]) / dx + (Gi[:, :, 1:] - Gi[:, :, :-1]) / dy


# --------------------------------------------------------------------------
# solver wiring  (simulation/set_simulator.py, time_step/TVD_RK3.py)
# --------------------------------------------------------------------------
class Solver:
    """Configured oracle for one grid: ``flux_func``, ``update_func``,
    ``advance_one_step`` and ``advance_func`` with the reference's
    signatures (set_simulator.py:20-125, 410-447)."""

    def __init__(self, mech, dim, dx, dy=None, bc=None, cfl=None, flux_config=None, transport_config=None,
                 time_scheme="TVD_RK3", source=None):
        self.time_scheme = time_scheme
        self.source = source  # source_config['self_defined_source_terms'](U, aux, dt, theta)
        self.m = mech
        self.dim = dim
        self.dx, self.dy = dx, dy
        self.bc = bc
        self.cfl = cfl
        self.last_iters = []
        # solver_{1D,2D}/flux.py set_flux_solver: flux splitting (LF) or
        # godunov with a Riemann solver, WENO5-JS reconstruction
        fc = flux_config or {"solver_type": "flux_splitting"}
        self.solver_type = fc["solver_type"]
        self.riemann = fc.get("riemann_solver", "HLLC")
        self.recon = fc.get("interface_reconstruction", "WENO5_JS")
        self.split = fc.get("split_method", "LF")
        self.transport = Transport(transport_config) if fc.get("viscosity", "off") == "on" else None

    def flux_func(self, U, aux, dx, dy, dt, theta=None):
        Up, Ap = boundary_conditions(self.m, U, aux, self.bc, theta)
        return self.padded_rhs(Up, Ap, dx, dy, dt)

    def padded_rhs(self, Up, Ap, dx, dy, dt):
        """dt * total_flux of ghost-padded arrays (set_simulator.py:26-47)."""
        if self.solver_type == "godunov":
            adv = godunov_flux(self.m, Up, Ap, dx, dy, self.riemann, self.recon)
        else:
            adv = total_flux(self.m, Up, Ap, dx, dy, self.recon, self.split)
        if self.transport is not None:  # NS_flux = advective + viscous (solver_2D/flux.py:117-118)
            return dt * (adv + viscous_flux(self.m, self.transport, Up, Ap, dx, dy))
        return dt * adv

    def update_func(self, U, aux):
        out, it = update_aux(self.m, U, aux, return_iters=True)
        self.last_iters.append(it)
        return out

    def rk3(self, U, aux, dx, dy, dt, theta, rhs_func=None, update_func=None):
        """TVD_RK3.py:5-12"""
        rhs_func = rhs_func or self.flux_func
        update_func = update_func or self.update_func
        U1 = U + rhs_func(U, aux, dx, dy, dt, theta)
        aux1 = update_func(U1, aux)
        U2 = 3 / 4 * U + 1 / 4 * (U1 + rhs_func(U1, aux1, dx, dy, dt, theta))
        aux2 = update_func(U2, aux1)
        U3 = 1 / 3 * U + 2 / 3 * (U2 + rhs_func(U2, aux2, dx, dy, dt, theta))
        aux3 = update_func(U3, aux2)
        return U3, aux3

    def rk2(self, U, aux, dx, dy, dt, theta, rhs_func=None, update_func=None):
        """RK2.py:5-12"""
        rhs_func = rhs_func or self.flux_func
        update_func = update_func or self.update_func
        dev = rhs_func(U, aux, dx, dy, dt, theta)
        U1 = U + dev
        aux1 = update_func(U1, aux)
        dev1 = rhs_func(U1, aux1, dx, dy, dt, theta)
        U2 = U + 1 / 2 * (dev + dev1)
        aux2 = update_func(U2, aux1)
        return U2, aux2

    def advance_one_step(self, U, aux, dx, dy, dt, theta=None):
        """set_simulator.py:73-122 (Lie splitting: time-stepped flux with the
        user source as set_advance_func composes it, chemistry, T)"""
        step = self.rk2 if self.time_scheme == "RK2" else self.rk3
        if self.source is None:
            U, aux = step(U, aux, dx, dy, dt, theta)
        elif self.solver_type == "flux_splitting":
            def rhs(U, aux, dx, dy, dt, theta=None):
                return self.flux_func(U, aux, dx, dy, dt, theta) + self.source(U, aux, dt, theta)
            U, aux = step(U, aux, dx, dy, dt, theta, rhs)
        else:
            U, aux = step(U, aux, dx, dy, dt, theta)
            U, aux = step(U, aux, dx, dy, dt, theta, lambda U, a, dx, dy, dt, th=None: self.source(U, a, dt, th))
        dU = reaction_source_terms(self.m, U, aux, dt)
        U = U + dU
        aux = self.update_func(U, aux)
        return U, aux

    def cfl_dt(self, U, aux):
        """CFL_1D / CFL_2D, set_simulator.py:420-443"""
        if U.ndim == 2:
            _, u, _, _, a = U_to_prim(self.m, U, aux)
            sx = np.abs(u) + a
            return self.cfl * np.min(self.dx / sx)
        _, u, v, _, _, a = U_to_prim(self.m, U, aux)
        sx = np.abs(u) + a
        sy = np.abs(v) + a
        return self.cfl * np.min(1 / (sx / self.dx + sy / self.dy))

    def advance_func(self, U, aux, t, theta=None):
        dt = self.cfl_dt(U, aux)
        U, aux = self.advance_one_step(U, aux, self.dx, self.dy, dt, theta)
        return U, aux, t + dt, dt


class SlabSolver:
    """The reference's parallel mode (``computation_config['is_parallel']``,
    set_simulator.py:20-47, 410-455, parallel/*.py) for P x slabs advanced in
    lockstep: lists of per-slab arrays in and out.  Each flux evaluation pads
    slab r from its neighbours (parallel_boundary_conditions); the LF wave
    speed and the temperature solve's stopping test are per slab (the pmapped
    body reduces over its own slab); the CFL dt is the minimum over the slabs
    (jax.lax.pmin).  ``thetas`` holds one theta per slab (PartitionDict)."""

    def __init__(self, mech, dim, dx, dy=None, bc=None, cfl=None, flux_config=None, transport_config=None):
        self.s = Solver(mech, dim, dx, dy, bc, cfl, flux_config, transport_config)
        self.m, self.bc = mech, bc

    def flux_func(self, Us, auxs, dx, dy, dt, thetas=None):
        thetas = thetas or [None] * len(Us)
        out = []
        for r in range(len(Us)):
            Up, Ap = parallel_boundary_conditions(self.m, Us, auxs, r, self.bc, thetas[r])
            out.append(self.s.padded_rhs(Up, Ap, dx, dy, dt))
        return out

    def rk3(self, Us, auxs, dx, dy, dt, thetas=None):
        """TVD_RK3.py:5-12 on every slab, one exchange per stage."""
        upd = self.s.update_func
        F = self.flux_func(Us, auxs, dx, dy, dt, thetas)
        U1 = [U + f for U, f in zip(Us, F)]
        A1 = [upd(U, a) for U, a in zip(U1, auxs)]
        F = self.flux_func(U1, A1, dx, dy, dt, thetas)
        U2 = [3 / 4 * U + 1 / 4 * (u1 + f) for U, u1, f in zip(Us, U1, F)]
        A2 = [upd(U, a) for U, a in zip(U2, A1)]
        F = self.flux_func(U2, A2, dx, dy, dt, thetas)
        U3 = [1 / 3 * U + 2 / 3 * (u2 + f) for U, u2, f in zip(Us, U2, F)]
        A3 = [upd(U, a) for U, a in zip(U3, A2)]
        return U3, A3

    def cfl_dt(self, Us, auxs):
        return np.min(np.array([self.s.cfl_dt(U, a) for U, a in zip(Us, auxs)]))

    def advance_func(self, Us, auxs, t, thetas=None):
        dt = self.cfl_dt(Us, auxs)
        Us, auxs = self.rk3(Us, auxs, self.s.dx, self.s.dy, dt, thetas)
        Us = [U + reaction_source_terms(self.m, U, a, dt) for U, a in zip(Us, auxs)]
        auxs = [self.s.update_func(U, a) for U, a in zip(Us, auxs)]
        return Us, auxs, t + dt, dt


# --------------------------------------------------------------------------
# initial-state builder (the examples' pattern)
# --------------------------------------------------------------------------
# --------------------------------------------------------------------------
# block-structured AMR step  (simulation/time_step/TVD_RK3.py:15-36 with the
# AMR block functions of simulation/set_simulator.py:37-42, 64-70, 97-113)
# --------------------------------------------------------------------------
def amr_flux_func(m, U, aux, dx, dy, dt, recon="WENO5_JS"):
    """set_simulator.py:37-40: per ghost-padded block [nv][bx+6][by+6],
    dt * total_flux padded back with three rows / columns of zeros (vmapped
    over the blocks, so the LF maxima are each block's own)."""
    out = np.zeros_like(U)
    for b in range(U.shape[0]):
        out[b, :, 3:-3, 3:-3] = dt * total_flux(m, U[b], aux[b], dx, dy, recon)
    return out


def amr_update_func(m, U, aux):
    """vmap(update_aux) (set_simulator.py:41): each block's temperature
    solve stops on its own max |res| (the batched while_loop)."""
    return np.stack([update_aux(m, np.ascontiguousarray(U[b]), aux[b]) for b in range(U.shape[0])])


def tvd_rk3_amr(m, amr, level, blk_data, dx, dy, dt, ref_blk_data, ref_blk_info, recon="WENO5_JS"):
    """TVD_RK3.advance_one_step_amr (TVD_RK3.py:15-36) with the block flux
    and update functions of set_rhs(is_amr=True).  ``amr`` is the block
    layer (``get_ghost_block_data``, ``update_external_boundary``);
    ``blk_data`` the coarser level's blocks, ``ref_blk_data`` this level's."""
    def rhs(U, aux):
        return amr_flux_func(m, U, aux, dx, dy, dt, recon)

    def upd(U, aux):
        return amr_update_func(m, U, aux)

    def back(U, aux):
        b = np.concatenate([U, aux], axis=1)[..., 3:-3, 3:-3]
        return amr.update_external_boundary(level, blk_data, np.ascontiguousarray(b), ref_blk_info)

    g = amr.get_ghost_block_data(ref_blk_data, ref_blk_info)
    U, aux = g[:, 0:-2], g[:, -2:]
    U1 = U + rhs(U, aux)
    aux1 = upd(U1, aux)
    g1 = amr.get_ghost_block_data(back(U1, aux1), ref_blk_info)
    U1, aux1 = g1[:, 0:-2], g1[:, -2:]
    U2 = 3 / 4 * U + 1 / 4 * (U1 + rhs(U1, aux1))
    aux2 = upd(U2, aux1)
    g2 = amr.get_ghost_block_data(back(U2, aux2), ref_blk_info)
    U2, aux2 = g2[:, 0:-2], g2[:, -2:]
    U3 = 1 / 3 * U + 2 / 3 * (U2 + rhs(U2, aux2))
    aux3 = upd(U3, aux2)
    return back(U3, aux3)


def amr_chemistry(m, blk, dt):
    """The detailed-chemistry part of the AMR advance_one_step
    (set_simulator.py:106-113): vmapped reaction_source_terms, U + dU and
    the blocks' update_aux, on unpadded blocks [nb][nv+2][bx][by]."""
    Ub, auxb = blk[:, 0:-2], blk[:, -2:]
    dU = np.stack([reaction_source_terms(m, np.ascontiguousarray(Ub[b]), auxb[b], dt) for b in range(Ub.shape[0])])
    Ub = Ub + dU
    auxb = amr_update_func(m, Ub, auxb)
    return np.concatenate([Ub, auxb], axis=1)


def advance_one_step_amr(m, amr, level, blk_data, dx, dy, dt, ref_blk_data, ref_blk_info, recon="WENO5_JS"):
    """One AMR step of the detailed-chemistry flux-splitting path (the
    advance_one_step of set_advance_func(is_amr=True), set_simulator.py:
    97-113): tvd_rk3_amr, then amr_chemistry."""
    blk = tvd_rk3_amr(m, amr, level, blk_data, dx, dy, dt, ref_blk_data, ref_blk_info, recon)
    return amr_chemistry(m, blk, dt)


def state_from_PTY(m, P, T, Y, vel=None):
    """rho = P/(R T), rhoE = rho h - P (+ kinetic), aux = [gamma, T]
    (examples/janc_basic_example1.ipynb, ``initial_conditions``)."""
    _, gamma, h, R, _ = get_thermo(m, T, Y)
    rho = P / (R * T)
    E = rho * h - P
    nd = T.ndim - 1
    if vel is None:
        vel = [np.zeros_like(T) for _ in range(nd)]
    for v in vel:
        E = E + 0.5 * rho * v ** 2
    U = np.concatenate([rho] + [rho * v for v in vel] + [E, rho * Y], axis=0)
    return U, np.concatenate([gamma, T], axis=0)


def stoich_Y(m, phi=1.0):
    """H2:O2:N2 = 2 phi : 1 : 3.76 by mole -> the 8 carried mass fractions."""
    W = {s: m.extra["MW"][i] for i, s in enumerate(m.species)}
    n = {"H2": 2.0 * phi, "O2": 1.0, "N2": 3.76}
    tot = sum(n[s] * W[s] for s in n)
    Y = np.zeros(m.ns - 1)
    Y[m.species.index("H2")] = n["H2"] * W["H2"] / tot
    Y[m.species.index("O2")] = n["O2"] * W["O2"] / tot
    return Y
