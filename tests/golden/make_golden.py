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

Usage:  python tests/golden/make_golden.py [--ref /path/to/JANC]
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    args = ap.parse_args()
    ref = args.ref
    _setup(ref)
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
