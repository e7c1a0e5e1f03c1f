"""Pin more of the NumPy oracle against golden vectors from the reference
JANC (janc_v2) itself, run by tests/golden/make_golden.py through the NumPy
stand-ins of JAX and Cantera:

* fsec_si.npz (group ``fsec``): flux_func of the reference's other flux
  options -- godunov_flux with HLLC and AUSMPW+ (riemann_solver/HLLC.py,
  riemann_solver/AUSMPW_plus.py), MUSCL reconstruction with LF splitting and
  with HLLC (reconstruction/MUSCL.py), and NS_flux with four laminar transport
  models and the Vreman LES closure (solver_{1D,2D}/flux.py viscous_flux,
  finite_difference/CENTRAL6.py, reconstruction/CENTRAL6.py,
  model/transport_model.py, model/LES/Verman.py) -- over two or three
  boundary sets each, plus Godunov steps (2D HLLC, 1D AUSMPW+);
* prim_si.npz (``prim``): U_to_prim (solver_{1D,2D}/aux_func.py:39-51);
* the initial-state builder of examples/janc_basic_example1.ipynb, whose
  reference output is the U0 / aux0 of the step fixtures;
* cfl2d_strip.npz (``cfl2d``): the 2D channel at config-1 spacing goes
  non-finite at CFL 0.1 in the reference itself;
* config0_cfl01_1000.npz (``long1d``) and channel128x64_200.npz (``mid2d``):
  long runs of the reference's Simulator.advance_func; the oracle is checked
  over their first steps here (the GPU tests run them to the end).

Bars: bitwise where the oracle restates the reference operation for
operation; 1e-15 relative L1 for the 1D AUSMPW+ flux, whose restatement
groups one product differently; 1e-12 for steps (pivoted LAPACK solve).
"""
import importlib.util
import os

import numpy as np
import pytest

from oracle import janc_oracle as jo

HERE = os.path.dirname(os.path.abspath(__file__))


def _make_golden():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


MG = _make_golden()
KEYS2 = ("left_boundary", "right_boundary", "bottom_boundary", "top_boundary")


def _load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name + ".npz"))


def _rel_l1(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.sum(np.abs(a - b)) / max(np.sum(np.abs(b)), 1e-300))


def _field_err(a, b, floor=1e-30):
    """Max over fields of the relative L1 error; a field whose reference L1
    sum is below ``floor`` is measured against ``floor`` instead (trace
    radicals at 1e-22, where the relative error says nothing)."""
    errs = [0.0]
    for i in range(b.shape[0]):
        den = np.sum(np.abs(b[i]))
        if den > 1e-30:
            errs.append(float(np.sum(np.abs(a[i] - b[i])) / max(den, floor)))
    return max(errs)


@pytest.fixture(scope="module")
def mech_si(mech_path):
    return jo.load_mechanism(mech_path)


@pytest.fixture(scope="module")
def mech_rdc(mech_path):
    return jo.load_mechanism(mech_path, {"P0": 10 * 101325, "T0": 300, "R0": 369, "x0": 0.08})


def _fsec_cases():
    cases = []
    for name, fc in MG.FSEC_FLUX.items():
        tcs = MG.FSEC_TRANSPORT if fc["viscosity"] == "on" else {"": None}
        for tname in tcs:
            if name != "AUSMPW_plus":  # the reference's 2D AUSMPW+ cannot run
                for bc in MG.FSEC_BC2:
                    cases.append(("2D", name, tname, bc))
            if not tname.startswith("les"):  # LES is 2D only in the reference
                for bc in MG.FSEC_BC1:
                    cases.append(("1D", name, tname, bc))
    return cases


@pytest.mark.parametrize("dim,name,tname,bc", _fsec_cases(),
                         ids=lambda v: v if isinstance(v, str) else "-".join(v))
def test_fsec_flux(dim, name, tname, bc, golden_dir, mech_si):
    g = _load(golden_dir, "fsec_si")
    key = ("f2d_" if dim == "2D" else "f1d_") + name + (("_" + tname) if tname else "") + "_" + "_".join(bc)
    fc = MG.FSEC_FLUX[name]
    tc = MG.FSEC_TRANSPORT[tname] if tname else None
    bcd = dict(zip(KEYS2, bc))
    theta = {"Pb": MG.FSEC_PB}
    with np.errstate(all="ignore"):
        if dim == "2D":
            b = _load(golden_dir, "bc2d_si")
            o = jo.Solver(mech_si, "2D", 1e-4, 2e-4, bcd, 0.5, flux_config=fc, transport_config=tc)
            r = o.flux_func(b["U"], b["aux"], 1e-4, 2e-4, 2e-8, theta)
        else:
            b = _load(golden_dir, "bc1d_si")
            dx = 0.1 / b["U"].shape[1]
            o = jo.Solver(mech_si, "1D", dx, None, bcd, 0.5, flux_config=fc, transport_config=tc)
            r = o.flux_func(b["U"], b["aux"], dx, None, 2e-8, theta)
    ref = g[key]
    # NaN where the reference has NaN (an outlet ghost state with a negative
    # reconstructed pressure), finite elsewhere
    np.testing.assert_array_equal(np.isnan(r), np.isnan(ref))
    if name == "AUSMPW_plus":
        a, b_ = np.nan_to_num(r), np.nan_to_num(ref)
        assert _field_err(a, b_) <= 1e-15, _field_err(a, b_)
    else:
        np.testing.assert_array_equal(r, ref)


def test_godunov_steps(golden_dir, mech_si):
    g = _load(golden_dir, "fsec_si")
    s2 = _load(golden_dir, "step2d_si")
    bc2 = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient",
           "bottom_boundary": "slip_wall", "top_boundary": "slip_wall"}
    o = jo.Solver(mech_si, "2D", float(s2["dx"]), float(s2["dy"]), bc2, 0.5, flux_config=MG.FSEC_FLUX["HLLC"])
    U, aux, t = s2["U0"], s2["aux0"], 0.0
    for step in range(1, 3):
        U, aux, t, _ = o.advance_func(U, aux, t)
        assert _field_err(U, g[f"step2d_HLLC_U_{step}"]) <= 1e-12
        assert _field_err(aux, g[f"step2d_HLLC_aux_{step}"]) <= 1e-12
    s1 = _load(golden_dir, "step1d_si")
    bc1 = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"}
    o = jo.Solver(mech_si, "1D", float(s1["dx"]), None, bc1, 0.5, flux_config=MG.FSEC_FLUX["AUSMPW_plus"])
    U, aux, t = s1["U0"], s1["aux0"], 0.0
    for step in range(1, 4):
        U, aux, t, _ = o.advance_func(U, aux, t)
        # the 1e-16 flux difference reaches the radicals H, O, OH, H2O2 whose
        # reference sums are 1e-22 .. 1e-13 (rho Y units): floor them at 1e-10
        # of the density sum
        assert _field_err(U, g[f"step1d_AUSMPW_plus_U_{step}"], 1e-10 * np.sum(g[f"step1d_AUSMPW_plus_U_{step}"][0])) <= 1e-12
        assert _field_err(aux, g[f"step1d_AUSMPW_plus_aux_{step}"]) <= 1e-12


def test_u_to_prim_bitwise(golden_dir, mech_si, mech_rdc):
    g = _load(golden_dir, "prim_si")
    for tag, fix, m, names in (("p2d", "bc2d_si", mech_si, ("rho", "u", "v", "Y", "p", "a")),
                               ("p1d", "bc1d_si", mech_si, ("rho", "u", "Y", "p", "a"))):
        b = _load(golden_dir, fix)
        out = jo.U_to_prim(m, b["U"], b["aux"])
        for n, v in zip(names, out):
            np.testing.assert_array_equal(v, g[f"{tag}_{n}"], err_msg=f"{tag} {n}")
    r = _load(golden_dir, "step2d_rdc")
    out = jo.U_to_prim(mech_rdc, r["U_3"], r["aux_3"])
    for n, v in zip(("rho", "u", "v", "Y", "p", "a"), out):
        np.testing.assert_array_equal(v, g[f"prdc_{n}"], err_msg=f"rdc {n}")


def state_inputs(golden_dir, which):
    """(P, T, Y) from which a step fixture's U0 / aux0 were built by the
    reference's state builder (make_golden._state): the pressures and
    temperatures are the stated constants (T as stored in aux0), Y the
    stoichiometric mixture of make_golden._stoich_Y."""
    if which == "config0_cfl05":
        g = _load(golden_dir, which)
        n = g["U0"].shape[1]
        P = np.full((1, n), 101325.0)
        P[:, :40] = 30 * 101325.0
        T = np.ascontiguousarray(g["aux0"][1:2])
        Y = np.ascontiguousarray(np.tile(MG._stoich_Y(1.0)[:, None], (1, n)))
        return g, P, T, Y
    g = _load(golden_dir, which)  # step2d_si: slab = first 3 columns
    nx, ny = g["U0"].shape[1:]
    P = np.full((1, nx, ny), 101325.0)
    P[:, :3] = 30 * 101325.0
    T = np.ascontiguousarray(g["aux0"][1:2])
    Y = np.ascontiguousarray(np.tile(MG._stoich_Y(1.0)[:, None, None], (1, nx, ny)))
    return g, P, T, Y


@pytest.mark.parametrize("which", ["config0_cfl05", "step2d_si"])
def test_state_from_PTY_bitwise(which, golden_dir, mech_si):
    g, P, T, Y = state_inputs(golden_dir, which)
    U, aux = jo.state_from_PTY(mech_si, P, T, Y)
    np.testing.assert_array_equal(U, g["U0"])
    np.testing.assert_array_equal(aux, g["aux0"])


def test_cfl2d_strip_blows_up_like_reference(golden_dir, mech_si):
    """The channel at config-1 spacing: the reference goes non-finite at
    CFL 0.1 within a few tens of steps; the oracle's steps 1 and 10 agree
    with it, and it fails at the same step."""
    g = _load(golden_dir, "cfl2d_strip")
    bc = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient",
          "bottom_boundary": "slip_wall", "top_boundary": "slip_wall"}
    d = float(g["dx"])
    bad_ref = int(g["cfl0.1_first_nonfinite_step"])
    assert 10 < bad_ref <= 100
    assert int(g["cfl0.05_first_nonfinite_step"]) == -1
    o = jo.Solver(mech_si, "2D", d, d, bc, 0.1)
    U, aux, t = g["U0"], g["aux0"], 0.0
    bad = -1
    with np.errstate(all="ignore"):
        for step in range(1, bad_ref + 1):
            U, aux, t, _ = o.advance_func(U, aux, t)
            if step in (1, 10):
                assert _field_err(U, g[f"cfl0.1_U_{step}"]) <= 1e-12
                assert _field_err(aux, g[f"cfl0.1_aux_{step}"]) <= 1e-12
            if not np.all(np.isfinite(U)):
                bad = step
                break
    assert bad == bad_ref


def test_config0_cfl01_first_steps(golden_dir, mech_si):
    """The 1000-step reference run of config 0 at CFL 0.1: the oracle's
    first 10 steps agree (the GPU tests follow it to step 1000)."""
    g = _load(golden_dir, "config0_cfl01_1000")
    bc = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"}
    o = jo.Solver(mech_si, "1D", float(g["dx"]), None, bc, float(g["cfl"]))
    U, aux, t = g["U0"], g["aux0"], 0.0
    for step in range(1, 11):
        U, aux, t, dt = o.advance_func(U, aux, t)
        assert abs(dt - g["dts"][step - 1]) <= 1e-13 * g["dts"][step - 1]
        if step in (1, 10):
            assert _field_err(U, g[f"U_{step}"]) <= 1e-12
            assert _field_err(aux, g[f"aux_{step}"]) <= 1e-12


def test_channel128x64_first_step(golden_dir, mech_si):
    g = _load(golden_dir, "channel128x64_200")
    bc = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient",
          "bottom_boundary": "slip_wall", "top_boundary": "slip_wall"}
    d = float(g["dx"])
    o = jo.Solver(mech_si, "2D", d, d, bc, float(g["cfl"]))
    U, aux, t, dt = o.advance_func(g["U0"], g["aux0"], 0.0)
    assert abs(dt - g["dts"][0]) <= 1e-13 * g["dts"][0]
    assert _field_err(U, g["U_1"]) <= 1e-12
    assert _field_err(aux, g["aux_1"]) <= 1e-12
