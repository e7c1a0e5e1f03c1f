"""Pin the NumPy oracle against golden vectors produced by running the
reference JANC (janc_v2) itself (see tests/golden/make_golden.py).

Bars: tables, thermo, temperature solve and the flux/boundary paths are
float64 operation-for-operation restatements, so they must agree to the last
bit (or within a few ulps where a libm ``log``/``pow`` enters).  Chemistry and
full steps go through a pivoted LAPACK solve whose internal order differs with
the array layout, so they are held to 1e-12 relative.
"""
import os

import numpy as np
import pytest

from oracle import janc_oracle as jo


def _load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name + ".npz"))


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    den = np.maximum(np.abs(b), 1e-300)
    return float(np.max(np.abs(a - b) / den))


def _rel_l1(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.sum(np.abs(a - b)) / max(np.sum(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def mech_si(mech_path):
    return jo.load_mechanism(mech_path)


@pytest.fixture(scope="module")
def mech_rdc(mech_path):
    return jo.load_mechanism(mech_path, {"P0": 10 * 101325, "T0": 300, "R0": 369, "x0": 0.08})


@pytest.mark.parametrize("which", ["si", "rdc"])
def test_tables_bitwise(which, golden_dir, mech_si, mech_rdc):
    g = _load(golden_dir, "tables_" + which)
    m = mech_si if which == "si" else mech_rdc
    t = m.tables()
    for k in g.files:
        assert t[k].shape == g[k].shape or np.squeeze(t[k]).shape == np.squeeze(g[k]).shape, k
        np.testing.assert_array_equal(np.squeeze(t[k]), np.squeeze(g[k]), err_msg=k)


def test_thermo_bitwise(golden_dir, mech_si):
    g = _load(golden_dir, "thermo_si")
    cp, gamma, h, R, dcp = jo.get_thermo(mech_si, g["T"], g["Y"])
    for name, a in (("cp", cp), ("gamma", gamma), ("h", h), ("R", R), ("dcp", dcp)):
        np.testing.assert_array_equal(a, g[name], err_msg=name)


@pytest.mark.parametrize("case", ["far", "near", "exact"])
def test_update_aux_bitwise(case, golden_dir, mech_si):
    g = _load(golden_dir, "update_aux_si")
    out = jo.update_aux(mech_si, g["U"], g["aux_in_" + case])
    np.testing.assert_array_equal(out, g["aux_out_" + case])


@pytest.mark.parametrize("dt", ["1e-09", "1e-08", "1e-07"])
def test_chemistry(dt, golden_dir, mech_si):
    g = _load(golden_dir, "chem_si")
    S = jo.reaction_source_terms(mech_si, g["U"], g["aux"], float(dt))
    ref = g["S_" + dt]
    assert _rel_l1(S, ref) < 1e-13
    scale = np.max(np.abs(ref), axis=1, keepdims=True) + 1e-300
    assert float(np.max(np.abs(S - ref) / scale)) < 1e-11


def test_flux_1d_bitwise(golden_dir, mech_si):
    g = _load(golden_dir, "step1d_si")
    bc = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"}
    s = jo.Solver(mech_si, "1D", float(g["dx"]), None, bc, 0.5)
    rhs = s.flux_func(g["U0"], g["aux0"], float(g["dx"]), None, 1e-7)
    np.testing.assert_array_equal(rhs, g["rhs0"])


@pytest.mark.parametrize("lb,rb", [("periodic", "periodic"), ("zero_gradient", "slip_wall"),
                                   ("pressure_outlet", "pressure_outlet"),
                                   ("no_slip_wall", "zero_gradient")])
def test_bc_1d(lb, rb, golden_dir, mech_si):
    g = _load(golden_dir, "bc1d_si")
    nx = g["U"].shape[1]
    s = jo.Solver(mech_si, "1D", 0.1 / nx, None, {"left_boundary": lb, "right_boundary": rb}, 0.5)
    rhs = s.flux_func(g["U"], g["aux"], 0.1 / nx, None, 2e-8, {"Pb": 101325.0 * 1.3})
    np.testing.assert_array_equal(rhs, g[f"rhs_{lb}_{rb}"])


COMBOS_2D = [("periodic", "periodic", "periodic", "periodic"),
             ("slip_wall", "zero_gradient", "slip_wall", "slip_wall"),
             ("pressure_outlet", "zero_gradient", "no_slip_wall", "pressure_outlet"),
             ("zero_gradient", "pressure_outlet", "pressure_outlet", "zero_gradient")]


@pytest.mark.parametrize("combo", COMBOS_2D)
def test_bc_2d(combo, golden_dir, mech_si):
    g = _load(golden_dir, "bc2d_si")
    bc = dict(zip(["left_boundary", "right_boundary", "bottom_boundary", "top_boundary"], combo))
    s = jo.Solver(mech_si, "2D", 1e-4, 2e-4, bc, 0.5)
    rhs = s.flux_func(g["U"], g["aux"], 1e-4, 2e-4, 2e-8, {"Pb": 101325.0 * 1.3})
    np.testing.assert_array_equal(rhs, g["rhs_" + "_".join(combo)])


def _check_state(U, aux, gU, gaux, tol):
    assert _rel_l1(U, gU) <= tol, _rel_l1(U, gU)
    assert _rel_l1(aux, gaux) <= tol, _rel_l1(aux, gaux)


def test_steps_1d(golden_dir, mech_si):
    g = _load(golden_dir, "step1d_si")
    bc = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"}
    s = jo.Solver(mech_si, "1D", float(g["dx"]), None, bc, 0.5)
    U, aux, t = g["U0"], g["aux0"], 0.0
    for step in range(1, 11):
        U, aux, t, dt = s.advance_func(U, aux, t)
        assert abs(dt - g["dts"][step - 1]) <= 1e-13 * g["dts"][step - 1]
        if f"U_{step}" in g.files:
            _check_state(U, aux, g[f"U_{step}"], g[f"aux_{step}"], 1e-12)


def test_steps_2d(golden_dir, mech_si):
    g = _load(golden_dir, "step2d_si")
    bc = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient",
          "bottom_boundary": "slip_wall", "top_boundary": "slip_wall"}
    dx, dy = float(g["dx"]), float(g["dy"])
    s = jo.Solver(mech_si, "2D", dx, dy, bc, 0.5)
    np.testing.assert_array_equal(s.flux_func(g["U0"], g["aux0"], dx, dy, 1e-8), g["rhs0"])
    U, aux, t = g["U0"], g["aux0"], 0.0
    for step in range(1, 4):
        U, aux, t, dt = s.advance_func(U, aux, t)
        _check_state(U, aux, g[f"U_{step}"], g[f"aux_{step}"], 1e-12)
    Ua, auxa = s.advance_one_step(g["U0"], g["aux0"], dx, dy, 2e-8)
    _check_state(Ua, auxa, g["U_adv_dt2e-8"], g["aux_adv_dt2e-8"], 1e-12)
    Ur, auxr = s.rk3(g["U0"], g["aux0"], dx, dy, 2e-8, None)
    np.testing.assert_array_equal(Ur, g["U_rk3_dt2e-8"])
    np.testing.assert_array_equal(auxr, g["aux_rk3_dt2e-8"])


def test_steps_2d_rdc(golden_dir, mech_rdc):
    g = _load(golden_dir, "step2d_rdc")
    bc = {"left_boundary": "periodic", "right_boundary": "periodic",
          "bottom_boundary": "rdc_injector", "top_boundary": "pressure_outlet"}
    dx, dy = float(g["dx"]), float(g["dy"])
    s = jo.Solver(mech_rdc, "2D", dx, dy, bc, 0.5)
    theta = {"Yinj": g["Yinj"], "Pb": float(g["Pb"])}
    np.testing.assert_array_equal(s.flux_func(g["U0"], g["aux0"], dx, dy, 1e-3, theta), g["rhs0"])
    U, aux, t = g["U0"], g["aux0"], 0.0
    for step in range(1, 4):
        U, aux, t, dt = s.advance_func(U, aux, t, theta)
        _check_state(U, aux, g[f"U_{step}"], g[f"aux_{step}"], 1e-12)


def test_config0_cfl05_blows_up_like_reference(golden_dir, mech_si):
    """Config 0 exactly as stated (2000 cells, 30 atm / 3000 K slab of fresh
    mixture, CFL 0.5): the reference's own step goes non-finite at the same
    step in the oracle, and the states before agree bitwise."""
    g = _load(golden_dir, "config0_cfl05")
    bc = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"}
    s = jo.Solver(mech_si, "1D", float(g["dx"]), None, bc, 0.5)
    U, aux, t = g["U0"], g["aux0"], 0.0
    first_bad = -1
    with np.errstate(all="ignore"):
        for step in range(1, 21):
            U, aux, t, dt = s.advance_func(U, aux, t)
            if f"U_{step}" in g.files:
                np.testing.assert_array_equal(U, g[f"U_{step}"])
                np.testing.assert_array_equal(aux, g[f"aux_{step}"])
            if not np.all(np.isfinite(U)):
                first_bad = step
                break
    assert first_bad == int(g["first_nonfinite_step"]) > 0
