"""GPU parity: every kernel against the reference's golden vectors and the
NumPy oracle, through the C ABI (janc_b200.Solver -> libjanc_b200.so).

Tolerances (float64):
* ``fp64_strict`` (built with -fmad=false, reference operation order): flux,
  boundaries, thermo and the temperature solve are compared bitwise; anything
  through exp/log/pow or the 8x8 solve (chemistry, full steps) to 1e-12
  relative L1 per field.
* ``fp64`` (FMA contraction): 1e-12 per kernel, full steps 1e-10 relative L1
  per field (the bar for the FP64 build).
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from janc_b200.solver import Solver  # noqa: E402
from oracle import janc_oracle as jo  # noqa: E402

RDC_ND = {"P0": 10 * 101325, "T0": 300, "R0": 369, "x0": 0.08}
BC1 = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"}
BC2 = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient",
       "bottom_boundary": "slip_wall", "top_boundary": "slip_wall"}
BC_RDC = {"left_boundary": "periodic", "right_boundary": "periodic",
          "bottom_boundary": "rdc_injector", "top_boundary": "pressure_outlet"}
PRECS = ["fp64_strict", "fp64"]


def G(golden_dir, name):
    return np.load(os.path.join(golden_dir, name + ".npz"))


def cuda(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


def rel_l1(a, b):
    return float(np.sum(np.abs(a - b)) / max(np.sum(np.abs(b)), 1e-300))


def field_err(a, b):
    """max over fields of the relative L1 error (rows with any mass)."""
    errs = []
    for i in range(a.shape[0]):
        den = np.sum(np.abs(b[i]))
        if den > 1e-30:
            errs.append(np.sum(np.abs(a[i] - b[i])) / den)
    return max(errs)


@pytest.fixture(scope="module")
def mech_path():
    from janc_b200.mechanism import DEFAULT_MECHANISM
    return DEFAULT_MECHANISM


@pytest.fixture(scope="module")
def omech(mech_path):
    return jo.load_mechanism(mech_path)


@pytest.mark.parametrize("prec", PRECS)
def test_thermo(prec, golden_dir):
    g = G(golden_dir, "thermo_si")
    s = Solver(1, 16, dx=1.0, boundary_config=BC1, precision=prec)
    outs = s.get_thermo(cuda(g["T"]), cuda(g["Y"]))
    for name, o in zip(("cp", "gamma", "h", "R", "dcp"), outs):
        a, b = host(o), g[name]
        if prec == "fp64_strict":
            np.testing.assert_array_equal(a, b, err_msg=name)
        else:
            assert np.max(np.abs(a - b) / np.abs(b)) < 1e-13, name


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("case", ["far", "near", "exact"])
def test_update_aux(prec, case, golden_dir):
    g = G(golden_dir, "update_aux_si")
    U = g["U"]
    s = Solver(1, U.shape[1], dx=1.0, boundary_config=BC1, precision=prec)
    out = host(s.update_aux(cuda(U), cuda(g["aux_in_" + case])))
    if prec == "fp64_strict":
        np.testing.assert_array_equal(out, g["aux_out_" + case])
    else:
        assert np.max(np.abs(out - g["aux_out_" + case]) / np.abs(g["aux_out_" + case])) < 1e-12


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("dt", ["1e-09", "1e-08", "1e-07"])
def test_chemistry(prec, dt, golden_dir):
    g = G(golden_dir, "chem_si")
    s = Solver(1, g["U"].shape[1], dx=1.0, boundary_config=BC1, precision=prec)
    S = host(s.reaction_source_terms(cuda(g["U"]), cuda(g["aux"]), float(dt)))
    ref = g["S_" + dt]
    assert field_err(S[3:], ref[3:]) < 1e-12
    np.testing.assert_array_equal(S[:3], 0.0)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("lb,rb", [("periodic", "periodic"), ("zero_gradient", "slip_wall"),
                                   ("pressure_outlet", "pressure_outlet"),
                                   ("no_slip_wall", "zero_gradient")])
def test_flux_1d_boundaries(prec, lb, rb, golden_dir):
    g = G(golden_dir, "bc1d_si")
    nx = g["U"].shape[1]
    s = Solver(1, nx, dx=0.1 / nx, boundary_config={"left_boundary": lb, "right_boundary": rb},
               precision=prec)
    r = host(s.flux_func(cuda(g["U"]), cuda(g["aux"]), 0.1 / nx, None, 2e-8, {"Pb": 101325.0 * 1.3}))
    ref = g[f"rhs_{lb}_{rb}"]
    if prec == "fp64_strict":
        np.testing.assert_array_equal(r, ref)
    else:
        assert field_err(r, ref) < 1e-12


COMBOS_2D = [("periodic", "periodic", "periodic", "periodic"),
             ("slip_wall", "zero_gradient", "slip_wall", "slip_wall"),
             ("pressure_outlet", "zero_gradient", "no_slip_wall", "pressure_outlet"),
             ("zero_gradient", "pressure_outlet", "pressure_outlet", "zero_gradient")]


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("combo", COMBOS_2D)
def test_flux_2d_boundaries(prec, combo, golden_dir):
    g = G(golden_dir, "bc2d_si")
    bc = dict(zip(["left_boundary", "right_boundary", "bottom_boundary", "top_boundary"], combo))
    nx, ny = g["U"].shape[1:]
    s = Solver(2, nx, ny, 1e-4, 2e-4, bc, precision=prec)
    r = host(s.flux_func(cuda(g["U"]), cuda(g["aux"]), 1e-4, 2e-4, 2e-8, {"Pb": 101325.0 * 1.3}))
    ref = g["rhs_" + "_".join(combo)]
    if prec == "fp64_strict":
        np.testing.assert_array_equal(r, ref)
    else:
        assert field_err(r, ref) < 1e-12


def _run_cfl(s, U, aux, nsteps, theta=None, cfl=0.5):
    Uo, auxo, dts = s.advance(cuda(U), cuda(aux), nsteps, cfl=cfl, theta=theta)
    return host(Uo), host(auxo), host(dts)


@pytest.mark.parametrize("prec", PRECS)
def test_steps_1d_golden(prec, golden_dir):
    g = G(golden_dir, "step1d_si")
    nx = g["U0"].shape[1]
    s = Solver(1, nx, dx=float(g["dx"]), boundary_config=BC1, precision=prec)
    r = host(s.flux_func(cuda(g["U0"]), cuda(g["aux0"]), float(g["dx"]), None, 1e-7))
    if prec == "fp64_strict":
        np.testing.assert_array_equal(r, g["rhs0"])
    tol = 1e-12 if prec == "fp64_strict" else 1e-10
    for n in (1, 2, 5, 10):
        U, aux, dts = _run_cfl(s, g["U0"], g["aux0"], n)
        assert field_err(U, g[f"U_{n}"]) < tol, (n, field_err(U, g[f"U_{n}"]))
        assert field_err(aux, g[f"aux_{n}"]) < tol
        np.testing.assert_allclose(dts, g["dts"][:n], rtol=tol)


@pytest.mark.parametrize("prec", PRECS)
def test_steps_2d_golden(prec, golden_dir):
    g = G(golden_dir, "step2d_si")
    nx, ny = g["U0"].shape[1:]
    dx, dy = float(g["dx"]), float(g["dy"])
    s = Solver(2, nx, ny, dx, dy, BC2, precision=prec)
    r = host(s.flux_func(cuda(g["U0"]), cuda(g["aux0"]), dx, dy, 1e-8))
    if prec == "fp64_strict":
        np.testing.assert_array_equal(r, g["rhs0"])
    tol = 1e-12 if prec == "fp64_strict" else 1e-10
    for n in (1, 3):
        U, aux, dts = _run_cfl(s, g["U0"], g["aux0"], n)
        assert field_err(U, g[f"U_{n}"]) < tol
        assert field_err(aux, g[f"aux_{n}"]) < tol
    Ua, auxa = s.advance_one_step(cuda(g["U0"]), cuda(g["aux0"]), dx, dy, 2e-8)
    assert field_err(host(Ua), g["U_adv_dt2e-8"]) < tol
    assert field_err(host(auxa), g["aux_adv_dt2e-8"]) < tol


@pytest.mark.parametrize("prec", PRECS)
def test_steps_rdc_golden(prec, golden_dir):
    g = G(golden_dir, "step2d_rdc")
    nx, ny = g["U0"].shape[1:]
    dx, dy = float(g["dx"]), float(g["dy"])
    s = Solver(2, nx, ny, dx, dy, BC_RDC, nondim_config=RDC_ND, precision=prec)
    theta = {"Yinj": g["Yinj"], "Pb": float(g["Pb"])}
    r = host(s.flux_func(cuda(g["U0"]), cuda(g["aux0"]), dx, dy, 1e-3, theta))
    if prec == "fp64_strict":
        np.testing.assert_array_equal(r, g["rhs0"])
    else:
        assert field_err(r, g["rhs0"]) < 1e-12
    tol = 1e-12 if prec == "fp64_strict" else 1e-10
    U, aux, dts = _run_cfl(s, g["U0"], g["aux0"], 3, theta)
    assert field_err(U, g["U_3"]) < tol
    assert field_err(aux, g["aux_3"]) < tol


def _c0_state(om, nx, slab):
    P = np.full((1, nx), 101325.0)
    T = np.full((1, nx), 300.0)
    Y = np.tile(jo.stoich_Y(om, 1.0)[:, None], (1, nx))
    P[:, :slab] = 30 * 101325.0
    T[:, :slab] = 3000.0
    return jo.state_from_PTY(om, P, T, Y)


@pytest.mark.parametrize("prec", PRECS)
def test_config0_cfl05_matches_reference_until_blowup(prec, golden_dir):
    """Config 0 exactly as stated (CFL 0.5): the reference's own step goes
    non-finite at step 17; the GPU path matches it at step 10 and flags the
    non-finite state through the status word by then."""
    g = G(golden_dir, "config0_cfl05")
    nx = g["U0"].shape[1]
    s = Solver(1, nx, dx=float(g["dx"]), boundary_config=BC1, precision=prec)
    tol = 1e-12 if prec == "fp64_strict" else 1e-10
    U, aux, _ = _run_cfl(s, g["U0"], g["aux0"], 10)
    assert field_err(U, g["U_10"]) < tol
    assert field_err(aux, g["aux_10"]) < tol
    assert s.status() == 0
    n_bad = int(g["first_nonfinite_step"])
    U, aux, _ = _run_cfl(s, g["U0"], g["aux0"], n_bad + 1)
    assert not np.all(np.isfinite(U))
    assert s.status() & 4


@pytest.mark.parametrize("prec", PRECS)
def test_oracle_1d_config0_size(prec, omech):
    """Config-0 grid (2000 cells, slab = first 2 %) at CFL 0.1, 40 steps, vs
    the oracle."""
    nx = 2000
    U0, aux0 = _c0_state(omech, nx, 40)
    o = jo.Solver(omech, "1D", 0.1 / nx, None, BC1, 0.1)
    U, aux, t = U0, aux0, 0.0
    for _ in range(40):
        U, aux, t, _dt = o.advance_func(U, aux, t)
    s = Solver(1, nx, dx=0.1 / nx, boundary_config=BC1, precision=prec)
    Ug, auxg, dts = _run_cfl(s, U0, aux0, 40, cfl=0.1)
    tol = 1e-12 if prec == "fp64_strict" else 1e-10
    assert field_err(Ug, U) < tol
    assert field_err(auxg, aux) < tol


@pytest.mark.parametrize("prec", PRECS)
def test_oracle_2d_ragged(prec, omech):
    """Ragged 2D grid (tile edges not aligned: 37 x 23) with a perturbed slab."""
    nx, ny = 37, 23
    rng = np.random.default_rng(7)
    P = np.full((1, nx, ny), 101325.0)
    T = np.full((1, nx, ny), 300.0)
    Y = np.tile(jo.stoich_Y(omech, 1.0)[:, None, None], (1, nx, ny))
    P[:, :4] = 30 * 101325.0
    T[:, :4] = 3000.0 * (1 + 0.05 * rng.uniform(-1, 1, (1, 4, ny)))
    U0, aux0 = jo.state_from_PTY(omech, P, T, Y)
    dx = dy = 1.953125e-4
    o = jo.Solver(omech, "2D", dx, dy, BC2, 0.5)
    U, aux, t = U0, aux0, 0.0
    for _ in range(4):
        U, aux, t, _dt = o.advance_func(U, aux, t)
    s = Solver(2, nx, ny, dx, dy, BC2, precision=prec)
    Ug, auxg, _ = _run_cfl(s, U0, aux0, 4)
    tol = 1e-12 if prec == "fp64_strict" else 1e-10
    assert field_err(Ug, U) < tol
    assert field_err(auxg, aux) < tol


@pytest.mark.parametrize("prec", PRECS)
def test_uniform_state_is_stationary(prec, omech):
    """A uniform gas at rest: the flux vanishes for periodic, slip and
    zero-gradient sides (size-independent property at a large grid)."""
    nx, ny = 256, 128
    P = np.full((1, nx, ny), 101325.0)
    T = np.full((1, nx, ny), 300.0)
    Y = np.tile(jo.stoich_Y(omech, 1.0)[:, None, None], (1, nx, ny))
    U0, aux0 = jo.state_from_PTY(omech, P, T, Y)
    for bc in (BC2, {"left_boundary": "periodic", "right_boundary": "periodic",
                     "bottom_boundary": "zero_gradient", "top_boundary": "zero_gradient"}):
        s = Solver(2, nx, ny, 1e-4, 1e-4, bc, precision=prec)
        r = host(s.flux_func(cuda(U0), cuda(aux0), 1e-4, 1e-4, 1e-8))
        assert np.max(np.abs(r)) <= 1e-9 * np.max(np.abs(U0))


@pytest.mark.parametrize("prec", PRECS)
def test_periodic_mass_conservation(prec, omech):
    """Periodic in x and y: total mass changes only by roundoff over steps."""
    nx, ny = 96, 64
    rng = np.random.default_rng(3)
    P = 101325.0 * (1 + 0.2 * rng.uniform(size=(1, nx, ny)))
    T = 300.0 + 900.0 * rng.uniform(size=(1, nx, ny))
    # the reference's periodic pad is node-periodic: column nx-1 is the same
    # node as column 0 (boundary_padding.py:6,22-23), so start consistent
    P[:, -1, :] = P[:, 0, :]
    T[:, -1, :] = T[:, 0, :]
    P[:, :, -1] = P[:, :, 0]
    T[:, :, -1] = T[:, :, 0]
    Y = np.tile(jo.stoich_Y(omech, 1.0)[:, None, None], (1, nx, ny))
    U0, aux0 = jo.state_from_PTY(omech, P, T, Y)
    per = {"left_boundary": "periodic", "right_boundary": "periodic",
           "bottom_boundary": "periodic", "top_boundary": "periodic"}
    s = Solver(2, nx, ny, 1e-4, 1e-4, per, precision=prec)
    U, aux, _ = _run_cfl(s, U0, aux0, 5)
    assert np.all(np.isfinite(U))
    assert s.status() == 0
    # conserved sum over the distinct nodes 0..nx-2 x 0..ny-2; the duplicate
    # column/row stays identical to its twin
    m0 = U0[0, :-1, :-1].sum()
    m1 = U[0, :-1, :-1].sum()
    assert abs(m1 - m0) / m0 < 1e-12
    np.testing.assert_array_equal(U[:, 0, :], U[:, -1, :])
    np.testing.assert_array_equal(U[:, :, 0], U[:, :, -1])


# --------------------------------------------------------------------------
# mixed precision: float32 flux arithmetic, float64 state / T-solve / chemistry
# bar: density relative L1 <= 1e-4, front position within 1 cell
# --------------------------------------------------------------------------
def _front(U, aux, omech, two_d):
    nY = 4 if two_d else 3
    Y = U[nY:] / U[0]
    p = U[0] * jo.get_R(omech, Y)[0] * aux[1]
    if two_d:
        return np.array([np.max(np.where(p[:, j] > 2 * 101325.0)[0], initial=-1) for j in range(p.shape[1])])
    return np.max(np.where(p > 2 * 101325.0)[0], initial=-1)


def _per_field(U, Uref, aux, auxref, omech, two_d):
    nY = 4 if two_d else 3
    out = {"rho": rel_l1(U[0], Uref[0]), "T": rel_l1(aux[1], auxref[1])}
    p = U[0] * jo.get_R(omech, U[nY:] / U[0])[0] * aux[1]
    pr = Uref[0] * jo.get_R(omech, Uref[nY:] / Uref[0])[0] * auxref[1]
    out["p"] = rel_l1(p, pr)
    for k in range(8):
        if np.sum(np.abs(Uref[nY + k])) > 1e-30:
            out[f"Y{k}"] = rel_l1(U[nY + k] / U[0], Uref[nY + k] / Uref[0])
    return out


def test_mixed_1d_config0_vs_oracle(omech):
    nx = 2000
    U0, aux0 = _c0_state(omech, nx, 40)
    o = jo.Solver(omech, "1D", 0.1 / nx, None, BC1, 0.1)
    U, aux, t = U0, aux0, 0.0
    for _ in range(100):
        U, aux, t, _dt = o.advance_func(U, aux, t)
    s = Solver(1, nx, dx=0.1 / nx, boundary_config=BC1, precision="mixed")
    Ug, auxg, _ = _run_cfl(s, U0, aux0, 100, cfl=0.1)
    errs = _per_field(Ug, U, auxg, aux, omech, False)
    assert errs["rho"] <= 1e-4, errs
    assert errs["p"] <= 1e-4 and errs["T"] <= 1e-4, errs
    assert abs(int(_front(Ug, auxg, omech, False)) - int(_front(U, aux, omech, False))) <= 1
    assert s.status() == 0


def test_mixed_2d_vs_oracle(omech):
    nx, ny = 37, 23
    rng = np.random.default_rng(7)
    P = np.full((1, nx, ny), 101325.0)
    T = np.full((1, nx, ny), 300.0)
    Y = np.tile(jo.stoich_Y(omech, 1.0)[:, None, None], (1, nx, ny))
    P[:, :4] = 30 * 101325.0
    T[:, :4] = 3000.0 * (1 + 0.05 * rng.uniform(-1, 1, (1, 4, ny)))
    U0, aux0 = jo.state_from_PTY(omech, P, T, Y)
    dx = dy = 1.953125e-4
    o = jo.Solver(omech, "2D", dx, dy, BC2, 0.1)
    U, aux, t = U0, aux0, 0.0
    for _ in range(10):
        U, aux, t, _dt = o.advance_func(U, aux, t)
    s = Solver(2, nx, ny, dx, dy, BC2, precision="mixed")
    Ug, auxg, _ = _run_cfl(s, U0, aux0, 10, cfl=0.1)
    errs = _per_field(Ug, U, auxg, aux, omech, True)
    assert errs["rho"] <= 1e-4 and errs["p"] <= 1e-4, errs
    assert np.max(np.abs(_front(Ug, auxg, omech, True) - _front(U, aux, omech, True))) <= 1


def test_mixed_rdc_flux_close_to_fp64(golden_dir):
    """The float32 flux against the reference's float64 flux_func on the RDC
    state (nondimensional, injector + outlet): relative L1 per field."""
    g = G(golden_dir, "step2d_rdc")
    nx, ny = g["U0"].shape[1:]
    dx, dy = float(g["dx"]), float(g["dy"])
    s = Solver(2, nx, ny, dx, dy, BC_RDC, nondim_config=RDC_ND, precision="mixed")
    theta = {"Yinj": g["Yinj"], "Pb": float(g["Pb"])}
    r = host(s.flux_func(cuda(g["U0"]), cuda(g["aux0"]), dx, dy, 1e-3, theta))
    assert field_err(r, g["rhs0"]) < 1e-5
    U, aux, _ = _run_cfl(s, g["U0"], g["aux0"], 3, theta)
    assert rel_l1(U[0], g["U_3"][0]) < 1e-6

