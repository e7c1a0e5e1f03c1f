"""Generate golden input/output vectors by executing the reference JANC
(``src/janc_v2``) itself.

JAX and Cantera are not installed in the build container, so the reference is
imported with the NumPy-backed stand-ins in ``tests/golden/refshim``
(``jax``, ``cantera``, ``jaxamr``, ``h5py``).  Everything else that runs is the
reference's own source, read from the reference checkout at generation time:
mechanism loading (``preprocess/load.py``), NASA7 thermo and the Halley
temperature solve (``model/thermo_model.py``), point-implicit chemistry
(``model/reaction_model.py``), ghost-cell fill (``boundary/``), LF splitting
and WENO5-JS (``solver_{1D,2D}/``), SSP-RK3 (``simulation/time_step``), and
``Simulator.advance_func`` with CFL time steps (``simulation/set_simulator.py``).
The rotating-detonation injector boundary is the user callable defined in
``examples/janc_basic_example2.ipynb``; its two functions are extracted from
the notebook JSON and executed unchanged.

Usage:  python tests/golden/make_golden.py --ref /path/to/JANC   (or JANC_REF=/path/to/JANC)
Writes ``tests/golden/*.npz`` (a few hundred KB in total).
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SPECIES8 = ["H2", "O2", "OH", "O", "H", "H2O", "HO2", "H2O2"]


def _setup(ref):
    sys.path.insert(0, os.path.join(HERE, "refshim"))
    sys.path.insert(0, os.path.join(ref, "src"))


def _sim_config(dim, mech, grid, bc, nondim=None, cfl=0.5, dt=None):
    cfg = {
        "dimension": dim,
        "grid_config": grid,
        "thermo_config": {"thermo_model": "nasa7", "mechanism_directory": mech},
        "reaction_config": {"is_detailed_chemistry": True, "mechanism_directory": mech},
        "flux_config": {"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS",
                        "split_method": "LF", "viscosity": "off"},
        "boundary_config": bc,
        "time_config": {"temporal_evolution_scheme": "TVD_RK3", "t_end": 1.0},
        "computation_config": {"output_settings": {"save_dt": 1.0, "results_path": "/tmp/_janc_golden.h5"}},
    }
    if dt is None:
        cfg["time_config"]["CFL"] = cfl
    else:
        cfg["time_config"]["dt"] = dt
    if nondim is not None:
        cfg["nondim_config"] = nondim
    return cfg


def C(x):
    """C-contiguous float64 array.  NumPy sums a C-contiguous (n, ...) array over axis 0
    row by row (sequentially); a Fortran-ordered one is summed pairwise.  All
    inputs are made C-contiguous so the species sums run in index order."""
    import jax.numpy as jnp
    return jnp.array(np.ascontiguousarray(np.asarray(x, dtype=np.float64)))


def _state(thermo_model, P, T, Y, vel=None):
    """Conserved state from (P, T, Y) with the reference's own get_thermo, as
    the examples build it: rho = P/(R T), rhoE = rho h - P (+ kinetic)."""
    P, T, Y = (np.ascontiguousarray(a) for a in (P, T, Y))
    _, gamma, h, R, _ = thermo_model.get_thermo(C(T), C(Y))
    rho = P / (R * T)
    E = rho * h - P
    nd = T.ndim - 1
    if vel is None:
        vel = [np.zeros_like(T) for _ in range(nd)]
    for v in vel:
        E = E + 0.5 * rho * v ** 2
    U = np.concatenate([rho] + [rho * v for v in vel] + [E, rho * Y], axis=0)
    aux = np.concatenate([gamma, T], axis=0)
    return np.ascontiguousarray(U), np.ascontiguousarray(aux)


def _stoich_Y(phi=1.0):
    # H2:O2:N2 = 2 phi : 1 : 3.76 by mole; molecular weights from the mechanism
    W = {"H2": 2.016, "O2": 31.998, "N2": 28.014}
    n = {"H2": 2.0 * phi, "O2": 1.0, "N2": 3.76}
    m = {k: n[k] * W[k] for k in n}
    tot = sum(m.values())
    Y = np.zeros(8)
    Y[0] = m["H2"] / tot
    Y[1] = m["O2"] / tot
    return Y


def _tables(thermo_model, reaction_model):
    rp = reaction_model.ReactionParams
    out = dict(
        species_M=thermo_model.species_M, Tcr=thermo_model.Tcr,
        cp_cof_low=thermo_model.cp_cof_low, cp_cof_high=thermo_model.cp_cof_high,
        dcp_cof_low=thermo_model.dcp_cof_low, dcp_cof_high=thermo_model.dcp_cof_high,
        h_cof_low=thermo_model.h_cof_low, h_cof_high=thermo_model.h_cof_high,
        h_cof_low_chem=reaction_model.h_cof_low_chem, h_cof_high_chem=reaction_model.h_cof_high_chem,
        s_cof_low=reaction_model.s_cof_low, s_cof_high=reaction_model.s_cof_high,
        logcof_low=reaction_model.logcof_low, logcof_high=reaction_model.logcof_high,
        A=rp["A"], B=rp["B"], EaR=rp["Ea/Ru"], vf=np.squeeze(rp["vf"]), vb=np.squeeze(rp["vb"]),
        third_body=np.squeeze(rp["third_body_coeffs"]), is_third_body=rp["is_third_body"],
        vsum=rp["vsum"],
    )
    return {k: np.asarray(v, dtype=np.float64) for k, v in out.items()}


def _load_notebook_injector(ref, thermo_model, U_to_prim):
    """Extract ``bottom_boundary`` and ``inj_model`` from the RDC notebook and
    execute them with the janc_v2 thermo module bound to the name ``thermo``."""
    import jax
    import jax.numpy as jnp
    nb = json.load(open(os.path.join(ref, "examples", "janc_basic_example2.ipynb")))
    src = None
    for c in nb["cells"]:
        s = "".join(c["source"])
        if "def bottom_boundary" in s and "def inj_model" in s:
            src = s
    assert src is not None
    start = src.index("def bottom_boundary")
    stop = src.index("##inlet boundary", start)
    code = src[start:stop].replace("from janc.solver.aux_func import U_to_prim", "")
    ns = {"jax": jax, "jnp": jnp, "thermo": thermo_model, "U_to_prim": U_to_prim}
    exec(compile(code, "janc_basic_example2.ipynb:bottom_boundary", "exec"), ns)
    return ns["bottom_boundary"], ns["inj_model"]


def gen_long1d(ref):
    """Config-0 physics (2000 cells, slab = first 2 %, slip wall left, zero
    gradient right) at CFL 0.1 for 1000 steps of the reference's own
    Simulator.advance_func; the state at steps 1, 10, 100 and 1000 and every
    step's dt.  About 45 minutes through the NumPy stand-ins."""
    from janc_v2.model import thermo_model
    from janc_v2.simulation import set_simulator
    mech = os.path.join(ref, "examples", "9sp-19r-H2-Air.yaml")
    t_start = time.time()
    nxc = 2000
    cfg = _sim_config("1D", mech, {"dx": 0.1 / nxc},
                      {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"}, cfl=0.1)
    sim = set_simulator.Simulator(cfg)
    P = np.full((1, nxc), 101325.0)
    T = np.full((1, nxc), 300.0)
    Y = np.tile(_stoich_Y(1.0)[:, None], (1, nxc))
    P[:, :40] = 30 * 101325.0
    T[:, :40] = 3000.0
    U0, aux0 = _state(thermo_model, P, T, Y)
    rec = {"U0": U0, "aux0": aux0, "dx": 0.1 / nxc, "cfl": 0.1}
    U, aux, t = C(U0), C(aux0), 0.0
    dts = []
    for step in range(1, 1001):
        U, aux, t, dt = sim.advance_func(U, aux, t, None)
        dts.append(float(dt))
        if step in (1, 10, 100, 1000):
            rec[f"U_{step}"] = np.asarray(U)
            rec[f"aux_{step}"] = np.asarray(aux)
            print(f"config 0, CFL 0.1: step {step}", time.time() - t_start, flush=True)
    rec["dts"] = np.array(dts)
    np.savez_compressed(os.path.join(HERE, "config0_cfl01_1000.npz"), **rec)


# flux options of SURVEY-row (f): the reference's godunov_flux with HLLC /
# AUSMPW+, MUSCL reconstruction, and NS_flux with its transport models and
# the Vreman LES closure (solver_{1D,2D}/flux.py, riemann_solver/,
# reconstruction/MUSCL.py, finite_difference/ and reconstruction/CENTRAL6.py,
# model/transport_model.py, model/LES/Verman.py)
FSEC_FLUX = {
    "HLLC": {"solver_type": "godunov", "interface_reconstruction": "WENO5_JS", "riemann_solver": "HLLC",
             "viscosity": "off"},
    "AUSMPW_plus": {"solver_type": "godunov", "interface_reconstruction": "WENO5_JS",
                    "riemann_solver": "AUSMPW_plus", "viscosity": "off"},
    "MUSCL_LF": {"solver_type": "flux_splitting", "interface_reconstruction": "MUSCL", "split_method": "LF",
                 "viscosity": "off"},
    "MUSCL_HLLC": {"solver_type": "godunov", "interface_reconstruction": "MUSCL", "riemann_solver": "HLLC",
                   "viscosity": "off"},
    "LF_visc": {"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS", "split_method": "LF",
                "viscosity": "on"},
}
FSEC_TRANSPORT = {
    "sutherland_pr_le": {"viscosity_model": "Sutherland", "thermal_conductivity_model": "Prandtl number",
                         "Pr": 0.72, "species_diffusivity_model": "Lewis number", "Le": 1.0},
    "sutherland_sc": {"viscosity_model": "Sutherland", "reference_viscosity": 1.8e-5,
                      "thermal_conductivity_model": "Prandtl number", "Pr": 0.7,
                      "species_diffusivity_model": "Schmidt number", "Sc": 0.5},
    "constant_all": {"viscosity_model": "constant", "dynamic_viscosity": 2e-5,
                     "thermal_conductivity_model": "constant", "thermal_conductivity": 0.05,
                     "species_diffusivity_model": "constant", "species_diffusivity": 3e-5},
    "constant_mu_le": {"viscosity_model": "constant", "dynamic_viscosity": 1.5e-5,
                       "thermal_conductivity_model": "constant", "thermal_conductivity": 0.04,
                       "species_diffusivity_model": "Lewis number", "Le": 0.8},
    "les_pr_le": {"viscosity_model": "Sutherland", "thermal_conductivity_model": "Prandtl number", "Pr": 0.72,
                  "species_diffusivity_model": "Lewis number", "Le": 1.0, "turbulence_model": "LES",
                  "LES_model": "Verman", "Pr_t": 0.9, "Le_t": 1.1},
    "les_constant": {"viscosity_model": "constant", "dynamic_viscosity": 2e-5,
                     "thermal_conductivity_model": "constant", "thermal_conductivity": 0.05,
                     "species_diffusivity_model": "constant", "species_diffusivity": 3e-5,
                     "turbulence_model": "LES", "LES_model": "Verman", "Pr_t": 0.85, "Sc_t": 0.7},
}
FSEC_BC2 = (("slip_wall", "zero_gradient", "slip_wall", "slip_wall"),
            ("pressure_outlet", "zero_gradient", "no_slip_wall", "pressure_outlet"),
            ("periodic", "periodic", "periodic", "periodic"))
FSEC_BC1 = (("zero_gradient", "slip_wall"), ("pressure_outlet", "no_slip_wall"))
FSEC_PB = 101325.0 * 1.3


def _fsec_flux(set_simulator, dim, mech, grid, bc, fc, tc, U, aux, dx, dy, dt):
    cfg = _sim_config(dim, mech, grid, bc)
    cfg["flux_config"] = fc
    if tc is not None:
        cfg["transport_config"] = tc
    set_simulator.Simulator(cfg)
    flux_func, _, _ = set_simulator.set_rhs(dim, cfg["reaction_config"])
    return np.asarray(flux_func(C(U), C(aux), dx, dy, dt, {"Pb": FSEC_PB}))


def gen_fsec(ref):
    """flux_func of the reference for every row-(f) flux option on the
    boundary-test states of bc1d_si / bc2d_si, and a few steps of the
    Godunov path (2D HLLC, 1D AUSMPW+) from the step fixtures' initial
    states.  The reference's 2D AUSMPW+ cannot run (its y faces take gamma
    from the x-face arrays, a shape mismatch), so it has no 2D fixture; LES
    is 2D only (Verman_1D is not in the reference's dictionary)."""
    from janc_v2.simulation import set_simulator
    mech = os.path.join(ref, "examples", "9sp-19r-H2-Air.yaml")
    t_start = time.time()
    out = {}
    b2 = np.load(os.path.join(HERE, "bc2d_si.npz"))
    U2, A2 = b2["U"], b2["aux"]
    dx2, dy2, dt2 = 1e-4, 2e-4, 2e-8
    for name, fc in FSEC_FLUX.items():
        if name == "AUSMPW_plus":
            continue
        tcs = FSEC_TRANSPORT if fc["viscosity"] == "on" else {"": None}
        for tname, tc in tcs.items():
            for bc in FSEC_BC2:
                bcd = dict(zip(("left_boundary", "right_boundary", "bottom_boundary", "top_boundary"), bc))
                key = "f2d_" + name + (("_" + tname) if tname else "") + "_" + "_".join(bc)
                out[key] = _fsec_flux(set_simulator, "2D", mech, {"dx": dx2, "dy": dy2}, bcd, fc, tc,
                                      U2, A2, dx2, dy2, dt2)
        print("2D", name, time.time() - t_start, flush=True)
    b1 = np.load(os.path.join(HERE, "bc1d_si.npz"))
    U1, A1 = b1["U"], b1["aux"]
    dx1, dt1 = 0.1 / U1.shape[1], 2e-8
    for name, fc in FSEC_FLUX.items():
        tcs = {k: v for k, v in FSEC_TRANSPORT.items() if not k.startswith("les")} \
            if fc["viscosity"] == "on" else {"": None}
        for tname, tc in tcs.items():
            for bc in FSEC_BC1:
                bcd = dict(zip(("left_boundary", "right_boundary"), bc))
                key = "f1d_" + name + (("_" + tname) if tname else "") + "_" + "_".join(bc)
                out[key] = _fsec_flux(set_simulator, "1D", mech, {"dx": dx1}, bcd, fc, tc, U1, A1, dx1, None, dt1)
        print("1D", name, time.time() - t_start, flush=True)
    # Godunov steps: advance_func of a configured Simulator (CFL 0.5)
    s2 = np.load(os.path.join(HERE, "step2d_si.npz"))
    bc2 = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient",
           "bottom_boundary": "slip_wall", "top_boundary": "slip_wall"}
    cfg = _sim_config("2D", mech, {"dx": float(s2["dx"]), "dy": float(s2["dy"])}, bc2)
    cfg["flux_config"] = FSEC_FLUX["HLLC"]
    sim = set_simulator.Simulator(cfg)
    U, aux, t = C(s2["U0"]), C(s2["aux0"]), 0.0
    for step in range(1, 3):
        U, aux, t, dt = sim.advance_func(U, aux, t, None)
        out[f"step2d_HLLC_U_{step}"] = np.asarray(U)
        out[f"step2d_HLLC_aux_{step}"] = np.asarray(aux)
    s1 = np.load(os.path.join(HERE, "step1d_si.npz"))
    bc1 = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"}
    cfg = _sim_config("1D", mech, {"dx": float(s1["dx"])}, bc1)
    cfg["flux_config"] = FSEC_FLUX["AUSMPW_plus"]
    sim = set_simulator.Simulator(cfg)
    U, aux, t = C(s1["U0"]), C(s1["aux0"]), 0.0
    for step in range(1, 4):
        U, aux, t, dt = sim.advance_func(U, aux, t, None)
        out[f"step1d_AUSMPW_plus_U_{step}"] = np.asarray(U)
        out[f"step1d_AUSMPW_plus_aux_{step}"] = np.asarray(aux)
    print("Godunov steps", time.time() - t_start, flush=True)
    np.savez_compressed(os.path.join(HERE, "fsec_si.npz"), **out)


def gen_prim(ref):
    """U_to_prim (solver_{1D,2D}/aux_func.py:39-51) of the reference on the
    boundary-test states (moving, non-uniform gas) and on the rotating-
    detonation initial state (nondimensional tables)."""
    from janc_v2.model import thermo_model
    from janc_v2.simulation import set_simulator
    from janc_v2.solver_1D import aux_func as aux1
    from janc_v2.solver_2D import aux_func as aux2
    mech = os.path.join(ref, "examples", "9sp-19r-H2-Air.yaml")
    out = {}
    set_simulator.Simulator(_sim_config("2D", mech, {"dx": 1e-4, "dy": 1e-4},
                                        {k: "slip_wall" for k in ("left_boundary", "right_boundary",
                                                                  "bottom_boundary", "top_boundary")}))
    b2 = np.load(os.path.join(HERE, "bc2d_si.npz"))
    for n, v in zip(("rho", "u", "v", "Y", "p", "a"), aux2.U_to_prim(C(b2["U"]), C(b2["aux"]))):
        out["p2d_" + n] = np.asarray(v)
    # the thermo module's broadcast shapes follow the last configured dimension
    set_simulator.Simulator(_sim_config("1D", mech, {"dx": 1e-4},
                                        {"left_boundary": "slip_wall", "right_boundary": "slip_wall"}))
    b1 = np.load(os.path.join(HERE, "bc1d_si.npz"))
    for n, v in zip(("rho", "u", "Y", "p", "a"), aux1.U_to_prim(C(b1["U"]), C(b1["aux"]))):
        out["p1d_" + n] = np.asarray(v)
    P0, T0, R0, x0 = 10 * 101325, 300, 369, 0.08
    cfg = _sim_config("2D", mech, {"dx": 1e-4 / x0, "dy": 1e-4 / x0},
                      {k: "slip_wall" for k in ("left_boundary", "right_boundary", "bottom_boundary",
                                                "top_boundary")},
                      nondim={"P0": P0, "T0": T0, "R0": R0, "x0": x0})
    set_simulator.Simulator(cfg)
    r = np.load(os.path.join(HERE, "step2d_rdc.npz"))
    for n, v in zip(("rho", "u", "v", "Y", "p", "a"), aux2.U_to_prim(C(r["U_3"]), C(r["aux_3"]))):
        out["prdc_" + n] = np.asarray(v)
    np.savez(os.path.join(HERE, "prim_si.npz"), **out)


def gen_cfl2d(ref):
    """The 2D channel's time-step limit in the reference itself: a 128 x 8
    strip at config-1 spacing (0.2 m / 1024), slab = first 21 columns at
    30 atm and 3000 K with a seeded +-5 % temperature perturbation, slip
    walls left, bottom and top, zero gradient right; up to 100 steps of
    Simulator.advance_func at CFL 0.1 and 0.05.  Records the first step
    whose state is non-finite (-1: none) and the states at steps 1 and 10."""
    from janc_v2.model import thermo_model
    from janc_v2.simulation import set_simulator
    mech = os.path.join(ref, "examples", "9sp-19r-H2-Air.yaml")
    t_start = time.time()
    nx, ny = 128, 8
    d = 0.2 / 1024
    rng = np.random.default_rng(7)
    P = np.full((1, nx, ny), 101325.0)
    T = np.full((1, nx, ny), 300.0)
    Y = np.tile(_stoich_Y(1.0)[:, None, None], (1, nx, ny))
    P[:, :21] = 30 * 101325.0
    T[:, :21] = 3000.0 * (1 + 0.05 * rng.uniform(-1, 1, (1, 21, ny)))
    bc = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient",
          "bottom_boundary": "slip_wall", "top_boundary": "slip_wall"}
    set_simulator.Simulator(_sim_config("2D", mech, {"dx": d, "dy": d}, bc, cfl=0.1))  # thermo tables
    U0, aux0 = _state(thermo_model, P, T, Y)
    rec = {"U0": U0, "aux0": aux0, "dx": d}
    for cfl in (0.1, 0.05):
        sim = set_simulator.Simulator(_sim_config("2D", mech, {"dx": d, "dy": d}, bc, cfl=cfl))
        U, aux, t = C(U0), C(aux0), 0.0
        bad = -1
        for step in range(1, 101):
            U, aux, t, dt = sim.advance_func(U, aux, t, None)
            if step in (1, 10):
                rec[f"cfl{cfl}_U_{step}"] = np.asarray(U)
                rec[f"cfl{cfl}_aux_{step}"] = np.asarray(aux)
            if not np.all(np.isfinite(np.asarray(U))):
                bad = step
                break
        rec[f"cfl{cfl}_first_nonfinite_step"] = np.array(bad)
        print(f"2D strip CFL {cfl}: first non-finite step {bad}", time.time() - t_start, flush=True)
    np.savez_compressed(os.path.join(HERE, "cfl2d_strip.npz"), **rec)


def gen_mid2d(ref):
    """A mid-size version of the 2D channel (config-1 spacing 0.2 m / 1024,
    128 x 64 cells, slab = first 21 columns at 30 atm / 3000 K with 8 seeded
    Gaussian temperature blobs of +-5 % and radius 2-6 cells,
    default_rng(1); slip walls left, bottom and top, zero gradient right) for
    200 steps of the reference's Simulator.advance_func at CFL 0.05; the
    state at steps 1, 20 and 200 and every dt."""
    from janc_v2.model import thermo_model
    from janc_v2.simulation import set_simulator
    mech = os.path.join(ref, "examples", "9sp-19r-H2-Air.yaml")
    t_start = time.time()
    nx, ny, slab = 128, 64, 21
    d = 0.2 / 1024
    rng = np.random.default_rng(1)
    P = np.full((1, nx, ny), 101325.0)
    T = np.full((1, nx, ny), 300.0)
    Y = np.tile(_stoich_Y(1.0)[:, None, None], (1, nx, ny))
    xs = np.arange(slab)[:, None]
    ys = np.arange(ny)[None, :]
    bump = np.zeros((slab, ny))
    for _ in range(8):
        a = rng.uniform(-0.05, 0.05)
        sig = rng.uniform(2.0, 6.0)
        cx = rng.uniform(0, slab)
        cy = rng.uniform(0, ny)
        bump += a * np.exp(-((xs - cx) ** 2 + (ys - cy) ** 2) / (2 * sig ** 2))
    P[0, :slab] = 30 * 101325.0
    T[0, :slab] = 3000.0 * (1 + bump)
    bc = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient",
          "bottom_boundary": "slip_wall", "top_boundary": "slip_wall"}
    sim = set_simulator.Simulator(_sim_config("2D", mech, {"dx": d, "dy": d}, bc, cfl=0.05))
    U0, aux0 = _state(thermo_model, P, T, Y)
    rec = {"U0": U0, "aux0": aux0, "dx": d, "cfl": 0.05}
    U, aux, t = C(U0), C(aux0), 0.0
    dts = []
    for step in range(1, 201):
        U, aux, t, dt = sim.advance_func(U, aux, t, None)
        dts.append(float(dt))
        if step in (1, 20, 200):
            rec[f"U_{step}"] = np.asarray(U)
            rec[f"aux_{step}"] = np.asarray(aux)
            print(f"128x64 channel: step {step}", time.time() - t_start, flush=True)
    rec["dts"] = np.array(dts)
    np.savez_compressed(os.path.join(HERE, "channel128x64_200.npz"), **rec)


def gen_amr(ref):
    """Block-AMR steps of the reference's own AMR_Simulator
    (set_simulator.py:496-532: advance_one_step_amr of TVD_RK3.py:15-36 with
    the vmapped block flux, update_aux and chemistry of set_simulator.py:
    37-42, 97-113), the external jaxamr block layer played by
    tests/golden/amr_blocks.py (a single level of blocks tiling a rectangle,
    zero-gradient mirror outside it).  Two layouts: 3 x 2 blocks of 20 x 20
    cells (each block two by two interior tiles of the kernel, one of them
    partial) for two steps, and 2 x 3 blocks of 7 x 9 cells for one step;
    SI units, dx = dy = 1e-4 m, dt = 1e-8 s; a 30 atm / 3000 K region with
    seeded +-5 % temperature blobs (default_rng(11)) over the block seams, a
    seeded velocity field of up to 50 m/s."""
    sys.path.insert(0, HERE)
    import amr_blocks
    import jaxamr
    from janc_v2.model import thermo_model
    from janc_v2.simulation import set_simulator
    jaxamr.amr.get_ghost_block_data = staticmethod(amr_blocks.get_ghost_block_data)
    jaxamr.amr.update_external_boundary = staticmethod(amr_blocks.update_external_boundary)
    mech = os.path.join(ref, "examples", "9sp-19r-H2-Air.yaml")
    cfg = _sim_config("2D", mech, {"dx": 1e-4, "dy": 1e-4},
                      {"left_boundary": "slip_wall", "right_boundary": "slip_wall",
                       "bottom_boundary": "slip_wall", "top_boundary": "slip_wall"})
    adv_amr, _ = set_simulator.AMR_Simulator(cfg)
    rng = np.random.default_rng(11)
    rec = {"dx": 1e-4, "dy": 1e-4, "dt": 1e-8}
    for name, nbx, nby, bx, by, nsteps in (("b20", 3, 2, 20, 20, 2), ("b7x9", 2, 3, 7, 9, 1)):
        nx, ny = nbx * bx, nby * by
        P = np.full((1, nx, ny), 101325.0)
        T = np.full((1, nx, ny), 300.0)
        Y = np.tile(_stoich_Y(1.0)[:, None, None], (1, nx, ny))
        hot = (np.arange(nx)[:, None] < int(0.45 * nx)) & (np.arange(ny)[None, :] < int(0.7 * ny))
        xs, ys = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
        bump = np.zeros((nx, ny))
        for _ in range(6):
            a, sig = rng.uniform(-0.05, 0.05), rng.uniform(1.5, 4.0)
            cx, cy = rng.uniform(0, nx), rng.uniform(0, ny)
            bump += a * np.exp(-((xs - cx) ** 2 + (ys - cy) ** 2) / (2 * sig ** 2))
        P[0][hot] = 30 * 101325.0
        T[0][hot] = 3000.0 * (1 + bump[hot])
        vel = [rng.uniform(-50.0, 50.0, (1, nx, ny)), rng.uniform(-50.0, 50.0, (1, nx, ny))]
        U0, aux0 = _state(thermo_model, P, T, Y, vel)
        grid = np.concatenate([U0, aux0], axis=0)
        blk = np.ascontiguousarray(amr_blocks.blocks_from_grid(grid, nbx, nby))
        info = amr_blocks.info(nbx, nby)
        rec[f"{name}_layout"] = np.array([nbx, nby, bx, by])
        rec[f"{name}_blk0"] = blk
        for s in range(1, nsteps + 1):
            blk = np.ascontiguousarray(np.asarray(adv_amr(1, C(blk), 1e-4, 1e-4, 1e-8, C(blk), info)))
            rec[f"{name}_blk{s}"] = blk
    np.savez_compressed(os.path.join(HERE, "amr_blocks.npz"), **rec)


GROUPS = {"long1d": gen_long1d, "fsec": gen_fsec, "prim": gen_prim, "cfl2d": gen_cfl2d, "mid2d": gen_mid2d,
          "amr": gen_amr}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("JANC_REF"),
                    help="checkout of the JANC repository (default: $JANC_REF)")
    ap.add_argument("--groups", default="core",
                    help="comma-separated fixture groups: core (the original set), " + ", ".join(GROUPS))
    args = ap.parse_args()
    ref = args.ref
    if not ref:
        ap.error("give the JANC checkout with --ref or JANC_REF")
    _setup(ref)
    groups = args.groups.split(",")
    for g in groups:
        if g != "core":
            GROUPS[g](ref)
    if "core" in groups:
        gen_core(ref)


def gen_core(ref):
    """The original fixture set (a few minutes)."""
    import jax.numpy as jnp
    from janc_v2.model import thermo_model, reaction_model
    from janc_v2.simulation import set_simulator
    from janc_v2.boundary import boundary as ref_boundary
    from janc_v2.solver_1D import aux_func as aux1
    from janc_v2.solver_2D import aux_func as aux2
    from janc_v2.simulation.time_step import time_step_dict

    mech = os.path.join(ref, "examples", "9sp-19r-H2-Air.yaml")
    rng = np.random.default_rng(20250407)
    t_start = time.time()

    # ---------------- 1D SI: tables, thermo, T solve, chemistry ----------------
    nx = 48
    cfg = _sim_config("1D", mech, {"dx": 0.1 / nx},
                      {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"})
    sim = set_simulator.Simulator(cfg)
    np.savez(os.path.join(HERE, "tables_si.npz"), **_tables(thermo_model, reaction_model))

    # thermo at temperatures spanning both NASA7 ranges and the switch point
    nT = 64
    T = np.concatenate([[250.0, 300.0, 999.999999, 1000.0, 1000.000001, 2500.0, 3400.0],
                        rng.uniform(260.0, 3500.0, nT - 7)])[None, :]
    Y = np.ascontiguousarray(rng.dirichlet(np.ones(9), nT).T[:8] * rng.uniform(0.2, 1.0, nT))
    cp, gamma, h, R, dcp = thermo_model.get_thermo(C(T), C(Y))
    np.savez(os.path.join(HERE, "thermo_si.npz"), T=T, Y=Y, cp=cp, gamma=gamma, h=h, R=R, dcp=dcp)

    # temperature solve: three guesses per state (far, near, exact)
    nS = 48
    Ts = rng.uniform(280.0, 3400.0, nS)[None, :]
    Ps = np.exp(rng.uniform(np.log(0.3e5), np.log(5e6), nS))[None, :]
    Ys = rng.dirichlet(np.ones(9), nS).T[:8] * rng.uniform(0.3, 1.0, nS)
    u = rng.uniform(-800, 800, nS)[None, :]
    U_s, aux_s = _state(thermo_model, Ps, Ts, Ys, [u])
    cases = {}
    for name, guess in (("far", Ts * rng.uniform(0.8, 1.2, Ts.shape)),
                        ("near", Ts * (1 + 1e-7 * rng.standard_normal(Ts.shape))),
                        ("exact", Ts.copy())):
        aux_in = np.concatenate([aux_s[0:1], guess])
        out = aux1.update_aux(C(U_s), C(aux_in))
        cases[f"aux_in_{name}"] = aux_in
        cases[f"aux_out_{name}"] = np.asarray(out)
    np.savez(os.path.join(HERE, "update_aux_si.npz"), U=U_s, **cases)

    # chemistry source at reacting states and three dt values
    nC = 40
    Tc = rng.uniform(900.0, 3300.0, nC)[None, :]
    Pc = np.exp(rng.uniform(np.log(0.5e5), np.log(5e6), nC))[None, :]
    Yc = np.zeros((8, nC))
    Y0 = _stoich_Y(1.0)
    for j in range(nC):
        burn = rng.uniform(0.0, 1.0)
        frac = rng.dirichlet(np.ones(8)) * rng.uniform(0.0, 0.05)
        Yc[:, j] = (1 - burn) * Y0
        Yc[5, j] += burn * (Y0[0] + Y0[1]) * 0.9
        Yc[:, j] += frac * (1 - Yc[:, j].sum()) * 0.5
    Yc[:, :4] = np.array([Y0] * 4).T  # fresh mixture, many species exactly 0
    Uc, auxc = _state(thermo_model, Pc, Tc, Yc)
    chem = {"U": Uc, "aux": auxc}
    for dt in (1e-9, 1e-8, 1e-7):
        S = reaction_model.reaction_source_terms(C(Uc), C(auxc), dt, None)
        chem[f"S_{dt:.0e}"] = np.asarray(S)
    np.savez(os.path.join(HERE, "chem_si.npz"), **chem)
    print("1D thermo/chem done", time.time() - t_start, flush=True)

    # ---------------- 1D full steps (config-0 physics on 48 cells) -------------
    P = np.full((1, nx), 101325.0)
    T = np.full((1, nx), 300.0)
    Y = np.tile(_stoich_Y(1.0)[:, None], (1, nx))
    P[:, :4] = 30 * 101325.0
    T[:, :4] = 3000.0
    U0, aux0 = _state(thermo_model, P, T, Y)
    rec = {"U0": U0, "aux0": aux0, "dx": 0.1 / nx}
    # flux_func on the initial state, and on a state with motion
    flux_func, update_func, _ = set_simulator.set_rhs("1D", cfg["reaction_config"])
    rec["rhs0"] = np.asarray(flux_func(C(U0), C(aux0), 0.1 / nx, None, 1e-7, None))
    U, aux, t = C(U0), C(aux0), 0.0
    dts = []
    for step in range(1, 11):
        U, aux, t, dt = sim.advance_func(U, aux, t, None)
        dts.append(float(dt))
        if step in (1, 2, 5, 10):
            rec[f"U_{step}"] = np.asarray(U)
            rec[f"aux_{step}"] = np.asarray(aux)
    rec["dts"] = np.array(dts)
    np.savez(os.path.join(HERE, "step1d_si.npz"), **rec)
    print("1D steps done", time.time() - t_start, flush=True)

    # config 0 at full size (2000 cells, slab = first 2 %, CFL 0.5): the
    # reference's own step goes non-finite after a few steps because the
    # first-order point-implicit chemistry burns a slab-edge cell in one step
    # and the Halley solve then diverges beyond the NASA7 range.
    nxc = 2000
    cfgc = _sim_config("1D", mech, {"dx": 0.1 / nxc},
                       {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"})
    simc = set_simulator.Simulator(cfgc)
    P = np.full((1, nxc), 101325.0)
    T = np.full((1, nxc), 300.0)
    Y = np.tile(_stoich_Y(1.0)[:, None], (1, nxc))
    P[:, :40] = 30 * 101325.0
    T[:, :40] = 3000.0
    U0, aux0 = _state(thermo_model, P, T, Y)
    rec = {"U0": U0, "aux0": aux0, "dx": 0.1 / nxc}
    U, aux, t = C(U0), C(aux0), 0.0
    first_bad = -1
    for step in range(1, 21):
        U, aux, t, dt = simc.advance_func(U, aux, t, None)
        if step in (1, 10):
            rec[f"U_{step}"] = np.asarray(U)
            rec[f"aux_{step}"] = np.asarray(aux)
        if not np.all(np.isfinite(np.asarray(U))):
            first_bad = step
            break
    rec["first_nonfinite_step"] = np.array(first_bad)
    np.savez_compressed(os.path.join(HERE, "config0_cfl05.npz"), **rec)
    print("config-0 CFL 0.5: first non-finite step", first_bad, time.time() - t_start, flush=True)

    # 1D boundary variants of flux_func on a moving, non-uniform state
    bvar = {}
    nxb = 24
    Pb = np.exp(rng.uniform(np.log(0.5e5), np.log(3e6), nxb))[None, :]
    Tb = rng.uniform(300, 3000, nxb)[None, :]
    Yb = np.tile(_stoich_Y(1.0)[:, None], (1, nxb)) * rng.uniform(0.7, 1.0, (1, nxb))
    ub = rng.uniform(-600, 600, nxb)[None, :]
    Ub, auxb = _state(thermo_model, Pb, Tb, Yb, [ub])
    bvar["U"], bvar["aux"] = Ub, auxb
    for lb, rb in (("periodic", "periodic"), ("zero_gradient", "slip_wall"),
                   ("pressure_outlet", "pressure_outlet"), ("no_slip_wall", "zero_gradient")):
        ref_boundary.set_boundary({"left_boundary": lb, "right_boundary": rb}, "1D")
        theta = {"Pb": 101325.0 * 1.3}
        r = flux_func(C(Ub), C(auxb), 0.1 / nxb, None, 2e-8, theta)
        bvar[f"rhs_{lb}_{rb}"] = np.asarray(r)
    np.savez(os.path.join(HERE, "bc1d_si.npz"), **bvar)

    # ---------------- 2D SI channel (config-1 physics, small grid) -------------
    nx2, ny2 = 20, 12
    Lx, Ly = 0.2 * nx2 / 1024, 0.05 * ny2 / 256
    cfg2 = _sim_config("2D", mech, {"dx": Lx / nx2, "dy": Ly / ny2},
                       {"left_boundary": "slip_wall", "right_boundary": "zero_gradient",
                        "bottom_boundary": "slip_wall", "top_boundary": "slip_wall"})
    sim2 = set_simulator.Simulator(cfg2)
    P = np.full((1, nx2, ny2), 101325.0)
    T = np.full((1, nx2, ny2), 300.0)
    Y = np.tile(_stoich_Y(1.0)[:, None, None], (1, nx2, ny2))
    P[:, :3] = 30 * 101325.0
    T[:, :3] = 3000.0 * (1 + 0.05 * rng.uniform(-1, 1, (1, 3, ny2)))
    U0, aux0 = _state(thermo_model, P, T, Y)
    rec = {"U0": U0, "aux0": aux0, "dx": Lx / nx2, "dy": Ly / ny2}
    flux2, _, _ = set_simulator.set_rhs("2D", cfg2["reaction_config"])
    rec["rhs0"] = np.asarray(flux2(C(U0), C(aux0), Lx / nx2, Ly / ny2, 1e-8, None))
    U, aux, t = C(U0), C(aux0), 0.0
    dts = []
    for step in range(1, 4):
        U, aux, t, dt = sim2.advance_func(U, aux, t, None)
        dts.append(float(dt))
        rec[f"U_{step}"] = np.asarray(U)
        rec[f"aux_{step}"] = np.asarray(aux)
    rec["dts"] = np.array(dts)
    # the explicit-dt step signature and the generic RK3 with the reference's
    # own rhs/update callables
    adv = set_simulator.set_advance_func("2D", cfg2["flux_config"], cfg2["reaction_config"],
                                         cfg2["time_config"], False, flux2, aux2.update_aux, None)
    Ua, auxa = adv(C(U0), C(aux0), Lx / nx2, Ly / ny2, 2e-8, None)
    rec["U_adv_dt2e-8"], rec["aux_adv_dt2e-8"] = np.asarray(Ua), np.asarray(auxa)
    Ur, auxr = time_step_dict["TVD_RK3"](C(U0), C(aux0), Lx / nx2, Ly / ny2, 2e-8,
                                         None, flux2, aux2.update_aux)
    rec["U_rk3_dt2e-8"], rec["aux_rk3_dt2e-8"] = np.asarray(Ur), np.asarray(auxr)
    np.savez(os.path.join(HERE, "step2d_si.npz"), **rec)
    print("2D SI done", time.time() - t_start, flush=True)

    # 2D boundary variants of flux_func on a moving, non-uniform state
    bvar = {}
    nxb, nyb = 14, 11
    Pb = np.exp(rng.uniform(np.log(0.5e5), np.log(3e6), (1, nxb, nyb)))
    Tb = rng.uniform(300, 3000, (1, nxb, nyb))
    Yb = np.tile(_stoich_Y(1.0)[:, None, None], (1, nxb, nyb)) * rng.uniform(0.7, 1.0, (1, nxb, nyb))
    ub = rng.uniform(-600, 600, (1, nxb, nyb))
    vb = rng.uniform(-600, 600, (1, nxb, nyb))
    Ub, auxb = _state(thermo_model, Pb, Tb, Yb, [ub, vb])
    bvar["U"], bvar["aux"] = Ub, auxb
    combos = (("periodic", "periodic", "periodic", "periodic"),
              ("slip_wall", "zero_gradient", "slip_wall", "slip_wall"),
              ("pressure_outlet", "zero_gradient", "no_slip_wall", "pressure_outlet"),
              ("zero_gradient", "pressure_outlet", "pressure_outlet", "zero_gradient"))
    for lb, rb, bb, tb in combos:
        ref_boundary.set_boundary({"left_boundary": lb, "right_boundary": rb,
                                   "bottom_boundary": bb, "top_boundary": tb}, "2D")
        theta = {"Pb": 101325.0 * 1.3}
        r = flux2(C(Ub), C(auxb), 1e-4, 2e-4, 2e-8, theta)
        bvar[f"rhs_{lb}_{rb}_{bb}_{tb}"] = np.asarray(r)
    np.savez(os.path.join(HERE, "bc2d_si.npz"), **bvar)
    print("2D BC done", time.time() - t_start, flush=True)

    # ---------------- 2D rotating-detonation setup (nondimensional) ------------
    P0, T0, R0, x0 = 10 * 101325, 300, 369, 0.08
    nondim = {"P0": P0, "T0": T0, "R0": R0, "x0": x0}
    nx3, ny3 = 16, 10
    dx3 = 1e-4 / x0
    # the injector needs the 2D U_to_prim and the nondim thermo tables
    cfg3 = _sim_config("2D", mech, {"dx": dx3, "dy": dx3},
                       {"left_boundary": "periodic", "right_boundary": "periodic",
                        "bottom_boundary": "slip_wall", "top_boundary": "pressure_outlet"},
                       nondim=nondim)
    set_simulator.Simulator(cfg3)  # sets nondim thermo so the injector sees it
    bottom_boundary, _ = _load_notebook_injector(ref, thermo_model, aux2.U_to_prim)
    cfg3["boundary_config"]["bottom_boundary"] = bottom_boundary
    sim3 = set_simulator.Simulator(cfg3)
    np.savez(os.path.join(HERE, "tables_rdc.npz"), **_tables(thermo_model, reaction_model))
    ratio = 1.0
    yH2 = (ratio / 8 * 0.232) / (1 + ratio / 8 * 0.232)
    yO2 = 0.232 / (1 + ratio / 8 * 0.232)
    Yinj = np.concatenate([[yH2, yO2], 1e-20 * np.ones(6)])
    theta = {"Yinj": np.tile(Yinj[:, None, None], (1, nx3, 1)), "Pb": 101325.0 / P0}
    Yenv = np.array([0, 0.232, 0, 0, 0, 0, 0, 0.0])
    Yfill = np.array([yH2, yO2, 0, 0, 0, 0, 0, 0.0])
    Y = np.tile(Yenv[:, None, None], (1, nx3, ny3))
    Y[:, : nx3 // 2, :4] = Yfill[:, None, None]
    T = np.full((1, nx3, ny3), 300.0 / T0)
    P = np.full((1, nx3, ny3), 101325.0 / P0)
    T[:, :3, :4] = 3000.0 / T0
    P[:, :3, :4] = 15 * 101325.0 / P0
    U0, aux0 = _state(thermo_model, P, T, Y)
    rec = {"U0": U0, "aux0": aux0, "dx": dx3, "dy": dx3, "Yinj": Yinj, "Pb": 101325.0 / P0}
    flux3, _, _ = set_simulator.set_rhs("2D", cfg3["reaction_config"])
    rec["rhs0"] = np.asarray(flux3(C(U0), C(aux0), dx3, dx3, 1e-3, theta))
    U, aux, t = C(U0), C(aux0), 0.0
    dts = []
    for step in range(1, 4):
        U, aux, t, dt = sim3.advance_func(U, aux, t, theta)
        dts.append(float(dt))
        rec[f"U_{step}"] = np.asarray(U)
        rec[f"aux_{step}"] = np.asarray(aux)
    rec["dts"] = np.array(dts)
    np.savez(os.path.join(HERE, "step2d_rdc.npz"), **rec)
    print("2D RDC done", time.time() - t_start, flush=True)


if __name__ == "__main__":
    main()
