"""The adjoint (reverse mode) of the 2D reacting step.

The checker is the torch float64 autograd twin of the reference's step
(oracle/janc_torch_twin.py, the stand-in for jax.grad of src/janc_v2, with
get_T's custom VJP and max / min splitting ties evenly), pinned itself to
the reference's golden steps and to central finite differences.  The
hand-written CUDA adjoint is compared with it, and with central finite
differences of the native forward.

Finite differences of this scheme only converge where no stencil sees
exactly uniform data: WENO5-JS with the reference's absolute eps = 1e-6
against split fluxes of order 1e8 is linear only for perturbations below
about 1e-11 relative there.  The finite-difference cases therefore start
from a state without exactly uniform regions.
"""
import numpy as np
import pytest

from oracle import janc_oracle as jo
from oracle import janc_torch_twin as tt

torch = pytest.importorskip("torch")

BC_SLIP = {k: "slip_wall" for k in ("left_boundary", "right_boundary", "bottom_boundary", "top_boundary")}
BC_MIX = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient",
          "bottom_boundary": "periodic", "top_boundary": "periodic"}
# outlets on a lo and a hi side, one per direction; the left one borders the
# hot region (its boundary cells can hold the alpha maximum)
BC_OUT = {"left_boundary": "pressure_outlet", "right_boundary": "zero_gradient",
          "bottom_boundary": "slip_wall", "top_boundary": "pressure_outlet"}
PB = 0.8 * 101325.0


@pytest.fixture(scope="module")
def omech():
    from janc_b200.mechanism import DEFAULT_MECHANISM
    return jo.load_mechanism(DEFAULT_MECHANISM)


def _fields(om, nx, ny, seed, noisy):
    rng = np.random.default_rng(seed)
    P = np.full((1, nx, ny), 101325.0)
    T = np.full((1, nx, ny), 300.0)
    P[:, :3] = 30 * 101325.0
    T[:, :3] = 3000.0 * (1 + 0.05 * rng.uniform(-1, 1, (1, 3, ny)))
    if noisy:
        T[:, 3:] *= 1 + 0.01 * rng.uniform(-1, 1, (1, nx - 3, ny))
    Y = np.tile(jo.stoich_Y(om, 1.0)[:, None, None], (1, nx, ny))
    return P, T, Y


# ------------------------------------------------------------------ CPU only
def test_twin_forward_matches_reference_steps(golden_dir, omech):
    """The twin's forward reproduces the reference's golden 2D steps."""
    import os
    g = np.load(os.path.join(golden_dir, "step2d_si.npz"))
    bc = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient",
          "bottom_boundary": "slip_wall", "top_boundary": "slip_wall"}
    tw = tt.Twin(omech, float(g["dx"]), float(g["dy"]), bc, 0.5)
    U, aux = torch.tensor(g["U0"]), torch.tensor(g["aux0"])
    for s in range(1, 4):
        dt = tt.cfl_dt(tw, U, aux)
        assert abs(float(dt) - float(g["dts"][s - 1])) <= 1e-13 * float(g["dts"][s - 1])
        U, aux = tt.advance_one_step(tw, U, aux, dt)
        ref = g[f"U_{s}"]
        for i in range(ref.shape[0]):
            den = np.abs(ref[i]).sum()
            if den > 1e-30:
                assert np.abs(U[i].numpy() - ref[i]).sum() / den < 1e-11


def _moving_state(om, nx, ny, seed):
    """A 2D state with the hot region of _fields at rest and Mach numbers up
    to 1.5 elsewhere: supersonic outflow through the right boundary cells
    for y < ny/2 and through the top ones for 3 <= x < nx/2, subsonic in- and
    outflow at the other boundary cells.  The hottest cell (1, ny/2) holds
    the maxima of |u| + a and |v| + a."""
    rng = np.random.default_rng(seed)
    P, T, Y = _fields(om, nx, ny, seed, noisy=True)
    T[0, 1, ny // 2] = 3500.0
    Mx = rng.uniform(-0.5, 0.5, (nx, ny))
    My = rng.uniform(-0.5, 0.5, (nx, ny))
    Mx[:3] = 0.0
    My[:3] = 0.0
    Mx[-1, :ny // 2] = 1.5
    My[3:nx // 2, -1] = 1.5
    return P, T, Y, Mx, My


def _with_velocity(U, aux, Mx, My, R):
    """U with velocities u = Mx a, v = My a at unchanged T (aux stays valid)."""
    rho, T, gamma = U[0], aux[1], aux[0]
    a = np.sqrt(gamma * R * T)
    u, v = Mx * a, My * a
    U = U.copy()
    U[1] = rho * u
    U[2] = rho * v
    U[3] = U[3] + 0.5 * rho * (u * u + v * v)
    return U


def test_twin_outlet_ghosts_match_oracle(omech):
    """The twin's pressure_outlet ghosts equal the oracle's (both branches,
    lo and hi sides in x and y)."""
    nx, ny = 12, 10
    P, T, Y, Mx, My = _moving_state(omech, nx, ny, 4)
    bc = {"left_boundary": "pressure_outlet", "right_boundary": "pressure_outlet",
          "bottom_boundary": "pressure_outlet", "top_boundary": "pressure_outlet"}
    tw = tt.Twin(omech, 1e-4, 1e-4, bc, 0.1, Pb=PB)
    U0, a0 = tt.state_from_PTY(tw, torch.tensor(P), torch.tensor(T), torch.tensor(Y))
    R = tt.get_R(tw, torch.tensor(Y)).numpy()[0]
    A = a0.numpy()
    U = _with_velocity(U0.numpy(), A, Mx, My, R)
    Up, Ap = tt.boundary_conditions(tw, torch.tensor(U), a0)
    Ur, Ar = jo.boundary_conditions(omech, U, A, bc, {"Pb": PB})
    # both branches occur on the right side
    mach = U[1, -1] / U[0, -1] / np.sqrt(A[0, -1] * R[-1] * A[1, -1])
    assert (mach > 1).any() and (mach < 1).any()
    for side in (np.s_[:, :3, 3:-3], np.s_[:, -3:, 3:-3], np.s_[:, 3:-3, :3], np.s_[:, 3:-3, -3:]):
        np.testing.assert_allclose(Up.numpy()[side], Ur[side], rtol=1e-14, atol=0)
        np.testing.assert_allclose(Ap.numpy()[side], Ar[side], rtol=1e-14, atol=0)


@pytest.mark.parametrize("bc", ["slip", "outlet"])
def test_twin_gradient_matches_finite_differences(omech, bc):
    nx, ny = 16, 12
    P, T, Y = _fields(omech, nx, ny, 5, noisy=True)
    tw = tt.Twin(omech, 1.953125e-4, 1.953125e-4, BC_SLIP if bc == "slip" else BC_OUT, 0.1, Pb=PB)
    Pt, Yt = torch.tensor(P), torch.tensor(Y)
    Tt = torch.tensor(T, requires_grad=True)
    lnA = torch.zeros(19, dtype=torch.float64, requires_grad=True)
    probe = (10, 4, 4, 4)
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
def _native(om, nx, ny, bc, P, T, Y, nsteps, cfl, probe, K, lnA=None):
    from janc_b200.adjoint import Trajectory, probe_trajectory
    from janc_b200.solver import Solver
    dx = dy = 1.953125e-4
    s = Solver(2, nx, ny, dx, dy, bc, precision="fp64")
    s.set_theta({"Pb": PB})
    traj = Trajectory(s, cfl, probe, checkpoint=K)
    cu = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    Tg = cu(T).requires_grad_()
    lg = torch.zeros(19, dtype=torch.float64, device="cuda", requires_grad=True) if lnA is None else lnA
    dts, pps = probe_trajectory(traj, cu(P), Tg, cu(Y), lg, nsteps)
    loss = (dts * pps).sum()
    loss.backward()
    return float(loss), Tg.grad.cpu().numpy(), lg.grad.cpu().numpy(), traj


def _twin(om, nx, ny, bc, P, T, Y, nsteps, cfl, probe):
    tw = tt.Twin(om, 1.953125e-4, 1.953125e-4, bc, cfl, Pb=PB)
    Tt = torch.tensor(T, requires_grad=True)
    lnA = torch.zeros(19, dtype=torch.float64, requires_grad=True)
    L, _, _ = tt.trajectory_loss(tw, torch.tensor(P), Tt, torch.tensor(Y), nsteps, probe, lnA)
    L.backward()
    return float(L), Tt.grad.numpy(), lnA.grad.numpy()


def _rel(a, b):
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize("bc,noisy", [(BC_SLIP, False), (BC_MIX, True), (BC_OUT, True)])
def test_adjoint_matches_autograd_twin(omech, bc, noisy):
    nx, ny, nsteps = 24, 16, 4
    P, T, Y = _fields(omech, nx, ny, 3, noisy)
    if bc is BC_OUT:
        # the alpha maxima start at a boundary cell of the left outlet, where
        # its ghosts' wave speeds tie with the cell's
        T[0, 0, ny // 2] = 3300.0
    probe = (14, 6, 4, 4)
    L, gT, gA, _ = _native(omech, nx, ny, bc, P, T, Y, nsteps, 0.1, probe, K=2)
    Lr, gTr, gAr = _twin(omech, nx, ny, bc, P, T, Y, nsteps, 0.1, probe)
    assert abs(L - Lr) <= 1e-12 * abs(Lr)
    assert _rel(gT, gTr) < 1e-8
    assert _rel(gA, gAr) < 1e-8


@pytest.mark.gpu
def test_adjoint_matches_finite_differences(omech):
    from janc_b200.adjoint import Trajectory
    from janc_b200.solver import Solver
    nx, ny, nsteps = 32, 24, 10
    P, T, Y = _fields(omech, nx, ny, 4, noisy=True)
    probe = (20, 10, 4, 4)
    L, gT, gA, traj = _native(omech, nx, ny, BC_SLIP, P, T, Y, nsteps, 0.1, probe, K=4)
    s = Solver(2, nx, ny, 1.953125e-4, 1.953125e-4, BC_SLIP, precision="fp64")
    t2 = Trajectory(s, 0.1, probe, checkpoint=nsteps)
    cu = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")

    def loss(Tn, dA):
        t2.set_log_A_offset(dA)
        U0, a0 = s.state_from_PTY(cu(P), cu(Tn), cu(Y))
        _, _, dts, pps, _ = t2.run(U0, a0, nsteps)
        return float((dts * pps).sum())
    rng = np.random.default_rng(11)
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
def test_adjoint_checkpoint_interval_does_not_change_gradient(omech):
    nx, ny, nsteps = 24, 16, 6
    P, T, Y = _fields(omech, nx, ny, 6, noisy=False)
    probe = (14, 6, 4, 4)
    L1, g1, a1, _ = _native(omech, nx, ny, BC_SLIP, P, T, Y, nsteps, 0.1, probe, K=nsteps)
    L2, g2, a2, _ = _native(omech, nx, ny, BC_SLIP, P, T, Y, nsteps, 0.1, probe, K=2)
    assert L1 == L2
    assert _rel(g2, g1) < 1e-13
    assert _rel(a2, a1) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("bc_name", ["mix", "outlet"])
@pytest.mark.parametrize("seed_kind", ["U", "aux", "species", "dt"])
def test_single_step_vjp_matches_twin(omech, seed_kind, bc_name):
    """One recorded step and jb_adjoint_step against the twin's reverse mode
    of the same step, for adjoint seeds on different outputs; "outlet": right
    and top pressure outlets with sub- and supersonic outflow (and inflow)
    through their boundary cells."""
    import ctypes
    from janc_b200.solver import Solver
    nx, ny = 24, 16
    dx = 1.953125e-4
    if bc_name == "mix":
        bc = BC_MIX
        P, T, Y = _fields(omech, nx, ny, 8, noisy=True)
    else:
        bc = {"left_boundary": "slip_wall", "right_boundary": "pressure_outlet",
              "bottom_boundary": "slip_wall", "top_boundary": "pressure_outlet"}
        P, T, Y, Mx, My = _moving_state(omech, nx, ny, 8)
    s = Solver(2, nx, ny, dx, dx, bc, precision="fp64")
    s.set_theta({"Pb": PB})
    L = s._lib
    cu = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    U0, a0 = s.state_from_PTY(cu(P), cu(T), cu(Y))
    if bc_name == "outlet":
        R = tt.get_R(tt.Twin(omech, dx, dx, bc, 0.1), torch.tensor(Y)).numpy()[0]
        U0 = cu(_with_velocity(U0.cpu().numpy(), a0.cpu().numpy(), Mx, My, R)).contiguous()
    assert L.jb_adjoint_reserve(s._h) == 0
    R = int(L.jb_record_doubles(s._h))
    rec = torch.empty(2 * R, dtype=torch.float64, device="cuda")
    rsl = torch.empty(13, dtype=torch.float64, device="cuda")
    dth = torch.empty(1, dtype=torch.float64, device="cuda")
    Uo, ao = torch.empty_like(U0), torch.empty_like(a0)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    assert L.jb_advance_ex(s._h, p(U0), p(a0), p(Uo), p(ao), 0.0, 0.1, 1, p(dth), None, p(rec), p(rsl), st) == 0
    rng = np.random.default_rng(2)
    WU = rng.standard_normal((12, nx, ny)) * (seed_kind in ("U", "species"))
    if seed_kind == "species":
        WU[:4] = 0.0
    WA = rng.standard_normal((2, nx, ny)) * (seed_kind == "aux")
    Wdt = 1e5 if seed_kind == "dt" else 0.0
    Ub, Ab = cu(WU).contiguous(), cu(WA).contiguous()
    dtb = cu([Wdt])
    lnAb = torch.zeros(19, dtype=torch.float64, device="cuda")
    assert L.jb_adjoint_step(s._h, p(rec), p(rsl), 0.1, p(Ub), p(Ab), p(dtb), None, p(lnAb), st) == 0
    # the twin's reverse mode of the same step from the same state
    tw = tt.Twin(omech, dx, dx, bc, 0.1, Pb=PB)
    Ut = U0.cpu().clone().requires_grad_()
    at = a0.cpu().clone().requires_grad_()
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
        # the two forwards differ by round-off (1e-13), which the adjoint of
        # the WENO weights amplifies by up to ~1e5 in places
        if name == "lnA":
            assert _rel(mine, ref) < 1e-7, name
            continue
        for f in range(ref.shape[0]):
            den = np.abs(ref[f]).sum()
            if den > 0:
                assert np.abs(mine[f] - ref[f]).sum() <= 1e-7 * den + 1e-14 * np.abs(ref).max() * ref[f].size, \
                    (name, f, _rel(mine[f], ref[f]))
