"""The adjoint with the rotating-detonation injector on the bottom side
(examples/janc_basic_example2.ipynb ``bottom_boundary`` + ``inj_model``) and
a pressure outlet on the top, periodic x: the nondimensional RDC state of
tests/golden/step2d_rdc.npz (made by the reference itself), whose bottom row
holds both injector branches (blocked where p >= 1, open elsewhere).

CPU: the autograd twin's injector ghosts equal the oracle's and its steps
the reference's golden steps.  GPU: one recorded step and jb_adjoint_step
against the twin's reverse mode for seeds on different outputs, and the
gradient of a 3-step probe-pressure loss with respect to the initial state
and ln A.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import janc_oracle as jo
from oracle import janc_torch_twin as tt

torch = pytest.importorskip("torch")

RDC_ND = {"P0": 10 * 101325, "T0": 300, "R0": 369, "x0": 0.08}
BC_RDC = {"left_boundary": "periodic", "right_boundary": "periodic",
          "bottom_boundary": "rdc_injector", "top_boundary": "pressure_outlet"}


@pytest.fixture(scope="module")
def rdc(golden_dir):
    return np.load(os.path.join(golden_dir, "step2d_rdc.npz"))


@pytest.fixture(scope="module")
def nmech():
    from janc_b200.mechanism import DEFAULT_MECHANISM
    return jo.load_mechanism(DEFAULT_MECHANISM, RDC_ND)


def _twin(nmech, g, cfl=0.5):
    return tt.Twin(nmech, float(g["dx"]), float(g["dy"]), BC_RDC, cfl, Pb=float(g["Pb"]), Yinj=g["Yinj"])


def _rel(a, b):
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))


# ------------------------------------------------------------------ CPU only
def test_twin_injector_matches_oracle_and_reference_steps(rdc, nmech):
    g = rdc
    U0, a0 = g["U0"], g["aux0"]
    _, _, _, _, p, _ = jo.U_to_prim(nmech, U0, a0)
    assert (p[0, :, 0] >= 1.0).any() and (p[0, :, 0] < 1.0).any()  # both branches
    Up, Ap = jo.boundary_conditions(nmech, U0, a0, BC_RDC, {"Yinj": g["Yinj"], "Pb": float(g["Pb"])})
    tw = _twin(nmech, g)
    Upt, Apt = tt.boundary_conditions(tw, torch.tensor(U0), torch.tensor(a0))
    sl = np.s_[:, 3:-3, :3]
    np.testing.assert_allclose(Upt.numpy()[sl], Up[sl], rtol=1e-14, atol=1e-300)
    np.testing.assert_allclose(Apt.numpy()[sl], Ap[sl], rtol=1e-14, atol=1e-300)
    U, A = torch.tensor(U0), torch.tensor(a0)
    for s in range(1, 4):
        dt = tt.cfl_dt(tw, U, A)
        assert abs(float(dt) - float(g["dts"][s - 1])) <= 1e-13 * float(g["dts"][s - 1])
        U, A = tt.advance_one_step(tw, U, A, dt)
        ref = g[f"U_{s}"]
        for i in range(ref.shape[0]):
            den = np.abs(ref[i]).sum()
            if den > 1e-30:
                assert np.abs(U[i].numpy() - ref[i]).sum() / den < 1e-12


# --------------------------------------------------------------------- GPU
def _state(g):
    """The golden RDC state with small seeded amounts of the six radical and
    product species (zero in the golden state).  At zero mass fraction the
    chemistry's clip (dY >= -Y) sits exactly at its kink, where the sign of a
    round-off-sized increment decides between a zero and a huge derivative
    in the reference's own formula; 1e-6 to 1e-5 of each keeps the
    derivative defined.  Both the native and the twin start from this state."""
    U, aux = g["U0"].copy(), g["aux0"]
    rng = np.random.default_rng(17)
    add = U[0:1] * rng.uniform(1e-6, 1e-5, (6,) + U.shape[1:])
    U[6:12] += add
    U[5:6] -= add.sum(axis=0, keepdims=True)  # taken from O2
    return U, aux


def _solver(g):
    from janc_b200.solver import Solver
    nx, ny = g["U0"].shape[1:]
    s = Solver(2, nx, ny, float(g["dx"]), float(g["dy"]), BC_RDC, nondim_config=RDC_ND, precision="fp64")
    s.set_theta({"Yinj": g["Yinj"], "Pb": float(g["Pb"])})
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("seed_kind", ["U", "aux", "species", "dt"])
def test_single_step_vjp_with_injector_matches_twin(rdc, nmech, seed_kind):
    g = rdc
    s = _solver(g)
    L = s._lib
    cu = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    U0n, a0n = _state(g)
    U0, a0 = cu(U0n), cu(a0n)
    nx, ny = g["U0"].shape[1:]
    cfl = 0.5
    assert L.jb_adjoint_reserve(s._h) == 0
    R = int(L.jb_record_doubles(s._h))
    rec = torch.empty(2 * R, dtype=torch.float64, device="cuda")
    rsl = torch.empty(13, dtype=torch.float64, device="cuda")
    dth = torch.empty(1, dtype=torch.float64, device="cuda")
    Uo, ao = torch.empty_like(U0), torch.empty_like(a0)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    assert L.jb_advance_ex(s._h, p(U0), p(a0), p(Uo), p(ao), 0.0, cfl, 1, p(dth), None, p(rec), p(rsl), st) == 0
    rng = np.random.default_rng(4)
    WU = rng.standard_normal((12, nx, ny)) * (seed_kind in ("U", "species"))
    if seed_kind == "species":
        WU[:4] = 0.0
    WA = rng.standard_normal((2, nx, ny)) * (seed_kind == "aux")
    Wdt = 1e3 if seed_kind == "dt" else 0.0
    Ub, Ab = cu(WU), cu(WA)
    dtb = cu([Wdt])
    lnAb = torch.zeros(19, dtype=torch.float64, device="cuda")
    assert L.jb_adjoint_step(s._h, p(rec), p(rsl), cfl, p(Ub), p(Ab), p(dtb), None, p(lnAb), st) == 0
    tw = _twin(nmech, g, cfl)
    Ut = torch.tensor(U0n, requires_grad=True)
    at = torch.tensor(a0n, requires_grad=True)
    lnA = torch.zeros(19, dtype=torch.float64, requires_grad=True)
    dt = tt.cfl_dt(tw, Ut, at)
    U1, a1 = tt.advance_one_step(tw, Ut, at, dt, lnA)
    obj = (U1 * torch.tensor(WU)).sum() + (a1 * torch.tensor(WA)).sum() + Wdt * dt
    gU, ga, gl = torch.autograd.grad(obj, (Ut, at, lnA))
    torch.cuda.synchronize()
    for name, mine, ref in (("U", Ub.cpu().numpy(), gU.numpy()), ("aux", Ab.cpu().numpy(), ga.numpy()),
                            ("lnA", lnAb.cpu().numpy(), gl.numpy())):
        if np.abs(ref).sum() == 0:
            assert np.abs(mine).sum() == 0, name
            continue
        if name == "lnA":
            assert _rel(mine, ref) < 1e-7, name
            continue
        for f in range(ref.shape[0]):
            den = np.abs(ref[f]).sum()
            if den > 0:
                assert np.abs(mine[f] - ref[f]).sum() <= 1e-7 * den + 1e-14 * np.abs(ref).max() * ref[f].size, \
                    (name, f, _rel(mine[f], ref[f]))
        # the boundary row (the injector cells) on its own
        den = np.abs(ref[:, :, 0]).sum()
        if den > 0:
            assert np.abs(mine[:, :, 0] - ref[:, :, 0]).sum() <= 1e-7 * den, (name, "bottom row")


@pytest.mark.gpu
def test_probe_loss_gradient_with_injector_matches_twin(rdc, nmech):
    """d/d(U0, aux0, ln A) of sum_n dt_n * mean p over a 4 x 3 probe after
    each of 3 CFL steps, through Trajectory (records, recomputation,
    jb_adjoint_step) against the twin."""
    from janc_b200.adjoint import Trajectory
    g = rdc
    s = _solver(g)
    cfl = 0.5
    probe = (6, 2, 4, 3)
    traj = Trajectory(s, cfl, probe, checkpoint=2)
    cu = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    U0n, a0n = _state(g)
    U0, a0 = cu(U0n), cu(a0n)
    _, _, dts, pps, ckpts = traj.run(U0, a0, 3)
    Ub, Ab, lnAb = traj.backward(ckpts, 3, pps, dts)
    tw = _twin(nmech, g, cfl)
    Ut = torch.tensor(U0n, requires_grad=True)
    at = torch.tensor(a0n, requires_grad=True)
    lnA = torch.zeros(19, dtype=torch.float64, requires_grad=True)
    U, a, Lt = Ut, at, 0.0
    for _ in range(3):
        dt = tt.cfl_dt(tw, U, a)
        U, a = tt.advance_one_step(tw, U, a, dt, lnA)
        Lt = Lt + dt * tt.probe_pressure(tw, U, a, probe)
    gU, ga, gl = torch.autograd.grad(Lt, (Ut, at, lnA))
    torch.cuda.synchronize()
    assert abs(float((dts * pps).sum()) - float(Lt)) <= 1e-12 * abs(float(Lt))
    assert _rel(Ub.cpu().numpy(), gU.numpy()) < 1e-8
    assert _rel(Ab.cpu().numpy(), ga.numpy()) < 1e-8
    assert _rel(lnAb.cpu().numpy(), gl.numpy()) < 1e-8
