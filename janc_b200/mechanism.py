"""Cantera-style YAML mechanism -> the constant tables the kernels use.

Restates JANC's loader (``src/janc_v2/preprocess/load.py:8-135``,
``read_reaction_mechanism`` and ``get_cantera_coeffs``; reference scales from
``preprocess/nondim.py:14-25``) without Cantera.  The Cantera 3.x conventions
that loader relies on are reproduced here:

* species order is the phase's ``species:`` list;
* molecular weights sum IUPAC conventional atomic weights
  (H 1.008, N 14.007, O 15.999, ...);
* NASA7 data ``[low, high]`` over ``[Tlow, Tmid, Thigh]``;
* the pre-exponential factor of a mechanism written in cm/mol is converted to
  SI-kmol by (1e-3)**(order-1) (order counts the third body), after which
  load.py:47 applies another (1e-3)**(order-1);
* Ea in cal/mol becomes J/kmol (x 4184) and load.py:49 divides by 1000;
* missing third-body efficiencies default to 1.

The arithmetic below follows load.py step for step so the tables equal the
reference's to the last bit.
"""
import ctypes
import os
from dataclasses import dataclass, field

import numpy as np
import yaml

RG = 8.314463
_ATOMIC_WEIGHT = {"H": 1.008, "He": 4.002602, "C": 12.011, "N": 14.007, "O": 15.999,
                  "Ar": 39.95}
_EA_TO_J_PER_KMOL = {"cal/mol": 4184.0, "kcal/mol": 4184000.0, "J/mol": 1000.0,
                     "kJ/mol": 1.0e6, "J/kmol": 1.0}

DEFAULT_MECHANISM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mechanisms",
                                 "9sp-19r-H2-Air.yaml")

NS_MAX, NR_MAX, NREAC_MAX = 9, 8, 19


@dataclass
class ReferenceScales:
    """nondim.set_nondim: P0, T0, R0, x0 and the derived scales."""
    P0: float = 1.0
    T0: float = 1.0
    R0: float = 1.0
    x0: float = 1.0

    @classmethod
    def from_config(cls, cfg):
        if cfg is None:
            return cls()
        return cls(cfg["P0"], cfg["T0"], cfg["R0"], cfg["x0"])

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
        return float(np.sqrt(self.P0 / self.rho0))

    @property
    def t0(self):
        return self.x0 / self.u0


@dataclass
class Mechanism:
    species: list
    scales: ReferenceScales
    molecular_weight: np.ndarray
    tables: dict = field(default_factory=dict)

    @property
    def ns(self):
        return len(self.species)

    @property
    def nr(self):
        return self.tables["vf"].shape[1]

    @property
    def nreac(self):
        return self.tables["vf"].shape[0]


def _split_side(side):
    species, third_body = {}, False
    for tok in side.split(" + "):
        tok = tok.strip()
        if tok == "M":
            third_body = True
            continue
        parts = tok.split()
        nu, name = (float(parts[0]), parts[1]) if len(parts) == 2 else (1.0, tok)
        species[name] = species.get(name, 0.0) + nu
    return species, third_body


def load(path=DEFAULT_MECHANISM, nondim_config=None):
    """Read a mechanism and build the reference's tables for the given
    non-dimensionalisation (None = SI)."""
    if os.path.splitext(path)[1].lower() != ".yaml":
        raise AssertionError("janc only read mech file with .yaml format")
    if not os.path.isfile(path):
        raise FileNotFoundError("No mechanism file detected in the specified directory.")
    sc = ReferenceScales.from_config(nondim_config)
    with open(path) as f:
        doc = yaml.safe_load(f)
    units = doc.get("units", {})
    cm_mol = (units.get("length", "m"), units.get("quantity", "kmol")) == ("cm", "mol")
    ea_factor = _EA_TO_J_PER_KMOL[units.get("activation-energy", "J/kmol")]
    phase = doc["phases"][0]
    species = list(phase["species"])
    elements = list(phase["elements"])
    by_name = {s["name"]: s for s in doc["species"]}
    ns = len(species)

    Tcr, low, high, mw = [], [], [], []
    for name in species:
        d = by_name[name]
        w = 0.0
        for el in elements:
            if el in d["composition"]:
                w += d["composition"][el] * _ATOMIC_WEIGHT[el]
        mw.append(w)
        th = d["thermo"]
        if th["model"] != "NASA7":
            raise NotImplementedError("only NASA7 thermo is supported")
        Tcr.append(th["temperature-ranges"][1])
        low.append(th["data"][0])
        high.append(th["data"][1])
    # get_cantera_coeffs (load.py:91-135)
    scale = np.array([[1, sc.T0, sc.T0 ** 2, sc.T0 ** 3, sc.T0 ** 4, 1 / sc.T0, 1]])
    c_lo = np.array(low, dtype=np.float64) * scale
    c_hi = np.array(high, dtype=np.float64) * scale
    species_M = np.array(mw) / (1000 * sc.M0)
    t = {}
    t["species_M"] = species_M
    t["Tcr"] = np.array(Tcr, dtype=np.float64) / sc.T0
    t["cp_cof_low"] = np.flip(c_lo[:, 0:5], axis=1) / species_M[:, None]
    t["cp_cof_high"] = np.flip(c_hi[:, 0:5], axis=1) / species_M[:, None]
    t["dcp_cof_low"] = t["cp_cof_low"][:, 0:-1] * np.array([[4, 3, 2, 1]])
    t["dcp_cof_high"] = t["cp_cof_high"][:, 0:-1] * np.array([[4, 3, 2, 1]])
    hw = np.array([[1 / 5, 1 / 4, 1 / 3, 1 / 2, 1, 1]])
    t["h_cof_low"] = np.flip(np.roll(c_lo[:, 0:6], 1, axis=1), axis=1) * hw / species_M[:, None]
    t["h_cof_high"] = np.flip(np.roll(c_hi[:, 0:6], 1, axis=1), axis=1) * hw / species_M[:, None]
    t["h_cof_low_chem"] = np.flip(np.roll(c_lo[:, 0:6], 1, axis=1), axis=1) * hw
    t["h_cof_high_chem"] = np.flip(np.roll(c_hi[:, 0:6], 1, axis=1), axis=1) * hw
    sw = np.array([[1 / 4, 1 / 3, 1 / 2, 1, 1]])
    t["s_cof_low"] = np.flip(np.concatenate([c_lo[:, -1:], c_lo[:, 1:5]], axis=1), axis=1) * sw
    t["s_cof_high"] = np.flip(np.concatenate([c_hi[:, -1:], c_hi[:, 1:5]], axis=1), axis=1) * sw
    t["logcof_low"] = c_lo[:, 0]
    t["logcof_high"] = c_hi[:, 0]

    # read_reaction_mechanism (load.py:8-88)
    reactions = doc.get("reactions", [])
    nreac = len(reactions)
    vf = np.zeros((nreac, ns))
    vb = np.zeros((nreac, ns))
    tb = np.zeros((nreac, ns))
    is_tb = np.zeros(nreac)
    A, B, Ea = [], [], []
    index = {n: i for i, n in enumerate(species)}
    for i, r in enumerate(reactions):
        eq = r["equation"]
        arrow = next(a for a in ("<=>", "=>", "=") if a in eq)
        lhs, rhs = eq.split(arrow)
        reac, m_on_left = _split_side(lhs)
        prod, _ = _split_side(rhs)
        typ = r.get("type", "elementary")
        if typ not in ("elementary", "three-body"):
            raise NotImplementedError(f"reaction type {typ!r} is not supported")
        three_body = typ == "three-body" or m_on_left
        for n, nu in reac.items():
            vf[i, index[n]] = nu
        for n, nu in prod.items():
            vb[i, index[n]] = nu
        order = sum(reac.values())
        if three_body:
            order += 1
            eff = r.get("efficiencies", {})
            for j, n in enumerate(species):
                tb[i, j] = eff.get(n, 1.0)
        is_tb[i] = 1.0 if np.any(tb[i, :] > 0) else 0.0
        rc = r["rate-constant"]
        a_si = float(rc["A"]) * (1.0e-3) ** (order - 1) if cm_mol else float(rc["A"])
        A.append(a_si * ((1e-3) ** (order - 1)))
        B.append(float(rc["b"]))
        Ea.append(float(rc["Ea"]) * ea_factor / 1000)
    keep = np.any(vf + vb != 0, axis=0)
    zero = np.all(vf + vb == 0, axis=0)
    if np.any(zero) and not np.all(zero[int(np.argmax(zero)):]):
        raise AssertionError("Inert species must be the last elements in species_list")
    vf = vf[:, keep]
    vb = vb[:, keep]
    vf_sum = np.sum(vf, axis=1)
    vb_sum = np.sum(vb, axis=1)
    A = np.array(A)
    B = np.array(B)
    Ea = np.array(Ea)
    t["A"] = (sc.t0 / sc.rho0) * (sc.T0 ** B) * ((sc.rho0 / sc.M0) ** vf_sum) * sc.M0 * A
    t["B"] = B
    t["EaR"] = Ea / (sc.e0 * sc.M0)
    t["vf"] = vf
    t["vb"] = vb
    t["third_body"] = tb * (sc.rho0 / sc.M0)
    t["is_third_body"] = is_tb
    t["vsum"] = vb_sum - vf_sum
    return Mechanism(species, sc, np.array(mw), t)


class MechParams(ctypes.Structure):
    """ctypes mirror of ``jb_mech_params`` (janc_b200/csrc/jb_types.h)."""
    _fields_ = [
        ("ns", ctypes.c_int), ("nr", ctypes.c_int), ("nreac", ctypes.c_int), ("pad_", ctypes.c_int),
        ("M", ctypes.c_double * NS_MAX), ("invM", ctypes.c_double * NS_MAX),
        ("Tcr", ctypes.c_double * NS_MAX),
        ("cp_lo", (ctypes.c_double * 5) * NS_MAX), ("cp_hi", (ctypes.c_double * 5) * NS_MAX),
        ("dcp_lo", (ctypes.c_double * 4) * NS_MAX), ("dcp_hi", (ctypes.c_double * 4) * NS_MAX),
        ("h_lo", (ctypes.c_double * 6) * NS_MAX), ("h_hi", (ctypes.c_double * 6) * NS_MAX),
        ("hc_lo", (ctypes.c_double * 6) * NS_MAX), ("hc_hi", (ctypes.c_double * 6) * NS_MAX),
        ("s_lo", (ctypes.c_double * 5) * NS_MAX), ("s_hi", (ctypes.c_double * 5) * NS_MAX),
        ("lg_lo", ctypes.c_double * NS_MAX), ("lg_hi", ctypes.c_double * NS_MAX),
        ("A", ctypes.c_double * NREAC_MAX), ("B", ctypes.c_double * NREAC_MAX),
        ("EaR", ctypes.c_double * NREAC_MAX), ("vsum", ctypes.c_double * NREAC_MAX),
        ("is_tb", ctypes.c_double * NREAC_MAX),
        ("vf", (ctypes.c_double * NR_MAX) * NREAC_MAX), ("vb", (ctypes.c_double * NR_MAX) * NREAC_MAX),
        ("dv", (ctypes.c_double * NR_MAX) * NREAC_MAX), ("tb", (ctypes.c_double * NS_MAX) * NREAC_MAX),
        ("T0", ctypes.c_double), ("pref", ctypes.c_double),
        # derived by jb_create
        ("lnA", ctypes.c_double * NREAC_MAX), ("tbinvM", (ctypes.c_double * NR_MAX) * NREAC_MAX),
        ("lnpref", ctypes.c_double), ("lnT0", ctypes.c_double),
        ("gen_ok", ctypes.c_int), ("tcr_uniform", ctypes.c_int),
    ]


def _fill(dst, arr):
    arr = np.asarray(arr, dtype=np.float64)
    if arr.ndim == 1:
        for i, v in enumerate(arr):
            dst[i] = float(v)
    else:
        for i in range(arr.shape[0]):
            for j in range(arr.shape[1]):
                dst[i][j] = float(arr[i, j])


def pack(mech):
    """Mechanism -> jb_mech_params (the kernels' by-value parameter block)."""
    if (mech.ns, mech.nr, mech.nreac) != (NS_MAX, NR_MAX, NREAC_MAX):
        raise NotImplementedError(
            f"the kernels are compiled for {NS_MAX} species / {NR_MAX} reactive / "
            f"{NREAC_MAX} reactions; got {mech.ns}/{mech.nr}/{mech.nreac}")
    t = mech.tables
    p = MechParams()
    p.ns, p.nr, p.nreac = mech.ns, mech.nr, mech.nreac
    _fill(p.M, t["species_M"])
    _fill(p.invM, 1 / t["species_M"])
    _fill(p.Tcr, t["Tcr"])
    for name, key in (("cp_lo", "cp_cof_low"), ("cp_hi", "cp_cof_high"), ("dcp_lo", "dcp_cof_low"),
                      ("dcp_hi", "dcp_cof_high"), ("h_lo", "h_cof_low"), ("h_hi", "h_cof_high"),
                      ("hc_lo", "h_cof_low_chem"), ("hc_hi", "h_cof_high_chem"),
                      ("s_lo", "s_cof_low"), ("s_hi", "s_cof_high"), ("lg_lo", "logcof_low"),
                      ("lg_hi", "logcof_high"), ("A", "A"), ("B", "B"), ("EaR", "EaR"),
                      ("vsum", "vsum"), ("is_tb", "is_third_body"), ("vf", "vf"), ("vb", "vb"),
                      ("tb", "third_body")):
        _fill(getattr(p, name), t[key])
    _fill(p.dv, t["vb"] - t["vf"])
    p.T0 = float(mech.scales.T0)
    p.pref = 101325 / mech.scales.P0
    return p


def stoichiometric_Y(mech, phi=1.0):
    """Mass fractions of H2:O2:N2 = 2 phi : 1 : 3.76 (by mole) for the carried
    species (the last, N2, is implicit)."""
    w = dict(zip(mech.species, mech.molecular_weight))
    n = {"H2": 2.0 * phi, "O2": 1.0, "N2": 3.76}
    tot = sum(n[s] * w[s] for s in n)
    Y = np.zeros(mech.ns - 1)
    Y[mech.species.index("H2")] = n["H2"] * w["H2"] / tot
    Y[mech.species.index("O2")] = n["O2"] * w["O2"] / tot
    return Y
