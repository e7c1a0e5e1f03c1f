"""The adjoint of the 1D reacting step (solver_1D/*: 11 fields, the CFL time
step CFL min dx / (|u| + a), set_simulator.py:420-427).

The checker is the 1D form of the torch float64 autograd twin
(oracle/janc_torch_twin.py), itself pinned here to the oracle's 1D steps
(whose 1D path is pinned to the reference's golden vectors) and to central
finite differences; the hand-written CUDA adjoint is compared with it and
with central finite differences of the native forward.
"""
import numpy as np
import pytest

from oracle import janc_oracle as jo
from oracle import janc_torch_twin as tt

torch = pytest.importorskip("torch")

DX = 5e-5
PB = 0.8 * 101325.0
BCS = {
    "slip_zg": {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"},
    "noslip_outlet": {"left_boundary": "no_slip_wall", "right_boundary": "pressure_outlet"},
    "periodic": {"left_boundary": "periodic", "right_boundary": "periodic"},
}


@pytest.fixture(scope="module")
def omech():
    from janc_b200.mechanism import DEFAULT_MECHANISM
    return jo.load_mechanism(DEFAULT_MECHANISM)


def _fields(om, n, seed, noisy=True, hot=6):
    rng = np.random.default_rng(seed)
    P = np.full((1, n), 101325.0)
    T = np.full((1, n), 300.0)
    P[:, :hot] = 30 * 101325.0
    T[:, :hot] = 3000.0 * (1 + 0.05 * rng.uniform(-1, 1, (1, hot)))
    if noisy:
        T[:, hot:] *= 1 + 0.01 * rng.uniform(-1, 1, (1, n - hot))
    Y = np.tile(jo.stoich_Y(om, 1.0)[:, None], (1, n))
    return P, T, Y


def _rel(a, b):
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))


# ------------------------------------------------------------------ CPU only
@pytest.mark.parametrize("bc", list(BCS))
def test_twin_1d_forward_matches_oracle(omech, bc):
    n = 60
    P, T, Y = _fields(omech, n, 1)
    theta = {"Pb": PB}
    U, aux = jo.state_from_PTY(omech, P, T, Y)
    o = jo.Solver(omech, "1D", DX, None, BCS[bc], 0.1)
    tw = tt.Twin(omech, DX, None, BCS[bc], 0.1, Pb=PB)
    Ut, at = tt.state_from_PTY(tw, torch.tensor(P), torch.tensor(T), torch.tensor(Y))
    assert np.array_equal(Ut.numpy(), U)
    t = 0.0
    for _ in range(3):
        U, aux, t, dt = o.advance_func(U, aux, t, theta)
        dtt = tt.cfl_dt(tw, Ut, at)
        assert abs(float(dtt) - dt) <= 1e-14 * dt
        Ut, at = tt.advance_one_step(tw, Ut, at, dtt)
    for f in range(U.shape[0]):
        den = np.abs(U[f]).sum()
        if den > 1e-30:
            assert np.abs(Ut[f].numpy() - U[f]).sum() / den < 1e-12, f


def test_twin_1d_gradient_matches_finite_differences(omech):
    n = 40
    P, T, Y = _fields(omech, n, 2)
    tw = tt.Twin(omech, DX, None, BCS["noslip_outlet"], 0.1, Pb=PB)
    Pt, Yt = torch.tensor(P), torch.tensor(Y)
    Tt = torch.tensor(T, requires_grad=True)
    lnA = torch.zeros(19, dtype=torch.float64, requires_grad=True)
    probe = (28, 0, 4, 1)
    L, _, _ = tt.trajectory_loss(tw, Pt, Tt, Yt, 3, probe, lnA)
    L.backward()
    rng = np.random.default_rng(9)
    h = 1e-6

    def loss(Tn, dA):
        with torch.no_grad():
            return float(tt.trajectory_loss(tw, Pt, torch.tensor(Tn), Yt, 3, probe, torch.tensor(dA))[0])
    for _ in range(2):
        d = rng.standard_normal(T.shape)
        d /= np.linalg.norm(d)
        fd = (loss(T * (1 + h * d), np.zeros(19)) - loss(T * (1 - h * d), np.zeros(19))) / (2 * h)
        ad = float((Tt.grad.numpy() * T * d).sum())
        assert abs(fd - ad) <= 1e-6 * abs(fd)
        e = rng.standard_normal(19)
        e /= np.linalg.norm(e)
        fd = (loss(T, h * e) - loss(T, -h * e)) / (2 * h)
        ad = float((lnA.grad.numpy() * e).sum())
        assert abs(fd - ad) <= 1e-5 * abs(fd)


# --------------------------------------------------------------------- GPU
def _native(bc, P, T, Y, nsteps, cfl, probe, K):
    from janc_b200.adjoint import Trajectory, probe_trajectory
    from janc_b200.solver import Solver
    s = Solver(1, P.shape[1], None, DX, None, bc, precision="fp64")
    s.set_theta({"Pb": PB})
    traj = Trajectory(s, cfl, probe, checkpoint=K)
    cu = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    Tg = cu(T).requires_grad_()
    lg = torch.zeros(19, dtype=torch.float64, device="cuda", requires_grad=True)
    dts, pps = probe_trajectory(traj, cu(P), Tg, cu(Y), lg, nsteps)
    loss = (dts * pps).sum()
    loss.backward()
    return float(loss), Tg.grad.cpu().numpy(), lg.grad.cpu().numpy(), s


def _twin(om, bc, P, T, Y, nsteps, cfl, probe):
    tw = tt.Twin(om, DX, None, bc, cfl, Pb=PB)
    Tt = torch.tensor(T, requires_grad=True)
    lnA = torch.zeros(19, dtype=torch.float64, requires_grad=True)
    L, _, _ = tt.trajectory_loss(tw, torch.tensor(P), Tt, torch.tensor(Y), nsteps, probe, lnA)
    L.backward()
    return float(L), Tt.grad.numpy(), lnA.grad.numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("bc", list(BCS))
def test_adjoint_1d_matches_autograd_twin(omech, bc):
    n, nsteps = 80, 5
    P, T, Y = _fields(omech, n, 3, noisy=(bc != "slip_zg"))
    if bc == "noslip_outlet":
        T[0, -1] = 600.0  # the outlet's boundary cell differs from its neighbour
    L, gT, gA, _ = _native(BCS[bc], P, T, Y, nsteps, 0.1, (50, 6), K=2)
    Lr, gTr, gAr = _twin(omech, BCS[bc], P, T, Y, nsteps, 0.1, (50, 0, 6, 1))
    assert abs(L - Lr) <= 1e-12 * abs(Lr)
    assert _rel(gT, gTr) < 1e-8, _rel(gT, gTr)
    assert _rel(gA, gAr) < 1e-8, _rel(gA, gAr)


@pytest.mark.gpu
def test_adjoint_1d_matches_finite_differences(omech):
    from janc_b200.adjoint import Trajectory
    n, nsteps = 120, 10
    P, T, Y = _fields(omech, n, 4, noisy=True)
    probe = (70, 0, 8, 1)
    L, gT, gA, s = _native(BCS["slip_zg"], P, T, Y, nsteps, 0.1, (70, 8), K=4)
    t2 = Trajectory(s, 0.1, probe, checkpoint=nsteps)
    cu = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")

    def loss(Tn, dA):
        t2.set_log_A_offset(dA)
        U0, a0 = s.state_from_PTY(cu(P), cu(Tn), cu(Y))
        _, _, dts, pps, _ = t2.run(U0, a0, nsteps)
        return float((dts * pps).sum())
    rng = np.random.default_rng(12)
    h = 1e-6
    for _ in range(3):
        d = rng.standard_normal(T.shape)
        d /= np.linalg.norm(d)
        fd = (loss(T * (1 + h * d), None) - loss(T * (1 - h * d), None)) / (2 * h)
        ad = float((gT * T * d).sum())
        assert abs(fd - ad) <= 1e-5 * abs(fd), (fd, ad)
        e = rng.standard_normal(19)
        e /= np.linalg.norm(e)
        fd = (loss(T, h * e) - loss(T, -h * e)) / (2 * h)
        ad = float((gA * e).sum())
        assert abs(fd - ad) <= 1e-5 * abs(fd), (fd, ad)


@pytest.mark.gpu
def test_adjoint_1d_checkpoint_interval_does_not_change_gradient(omech):
    n, nsteps = 64, 6
    P, T, Y = _fields(omech, n, 6, noisy=False)
    L1, g1, a1, _ = _native(BCS["slip_zg"], P, T, Y, nsteps, 0.1, (40, 4), K=nsteps)
    L2, g2, a2, _ = _native(BCS["slip_zg"], P, T, Y, nsteps, 0.1, (40, 4), K=2)
    assert L1 == L2
    assert _rel(g2, g1) < 1e-13
    assert _rel(a2, a1) < 1e-13
