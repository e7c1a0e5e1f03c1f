"""MUSCL interface reconstruction (reconstruction/MUSCL.py: minmod-limited,
kappa = 1/3, beta = 1) on the flux-splitting and Godunov paths.

CPU: the oracle's restatement reproduces linear data exactly, keeps face
values between their neighbours (TVD) and falls back to first order at an
extremum; these identities pin it without the reference.
GPU (through the C ABI): flux_func and RK steps against the oracle with
``interface_reconstruction: MUSCL``.  Tolerances: ``fp64_strict`` 1e-13
relative L1 per field for one flux and 1e-12 over steps; ``fp64`` 1e-12
and 1e-10; ``mixed`` (float32 reconstruction) 1e-4 per field and 1e-6 on
the density against the fp64 build.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import janc_oracle as jo  # noqa: E402

FC = {
    "LF": {"solver_type": "flux_splitting", "interface_reconstruction": "MUSCL", "split_method": "LF",
           "viscosity": "off"},
    "HLLC": {"solver_type": "godunov", "interface_reconstruction": "MUSCL", "riemann_solver": "HLLC",
             "viscosity": "off"},
    "AUSMPW_plus": {"solver_type": "godunov", "interface_reconstruction": "MUSCL",
                    "riemann_solver": "AUSMPW_plus", "viscosity": "off"},
}
BC2 = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient",
       "bottom_boundary": "slip_wall", "top_boundary": "slip_wall"}


@pytest.fixture(scope="module")
def omech():
    from janc_b200.mechanism import DEFAULT_MECHANISM
    return jo.load_mechanism(DEFAULT_MECHANISM)


def field_err(a, b):
    errs = []
    for i in range(a.shape[0]):
        den = np.sum(np.abs(b[i]))
        if den > 1e-30:
            errs.append(np.sum(np.abs(a[i] - b[i])) / den)
    return max(errs)


# ---------------------------------------------------------------- CPU
def test_flux_config_accepts_muscl():
    from janc_b200.solver import flux_scheme
    for k, fc in FC.items():
        assert flux_scheme(fc) == k


def test_oracle_muscl_linear_exact():
    """Faces of cells 1 .. n+4: face i of the output sits at padded x = i + 2.5."""
    x = np.arange(16.0)
    q = np.stack([2.0 * x + 1.0, -0.5 * x + 3.0])[:, :, None] * np.ones((1, 1, 10))
    for left in (True, False):
        r = jo._muscl(q, 1, 2, left)
        faces = np.arange(r.shape[1]) + 2.5
        assert r.shape == (2, 11, 4)
        assert np.allclose(r[0], (2.0 * faces + 1.0)[:, None])
        assert np.allclose(r[1], (-0.5 * faces + 3.0)[:, None])


def test_oracle_muscl_tvd_and_extrema():
    rng = np.random.default_rng(2)
    q = np.cumsum(rng.uniform(0.0, 1.0, 40))[None, :]  # monotone increasing
    L = jo._muscl(q, 1, None, True)[0]
    R = jo._muscl(q, 1, None, False)[0]
    # face f (padded f + 2.5) lies between cells f+2 and f+3
    lo, hi = q[0, 2:-3], q[0, 3:-2]
    assert np.all(L >= lo - 1e-12) and np.all(L <= hi + 1e-12)
    assert np.all(R >= lo - 1e-12) and np.all(R <= hi + 1e-12)
    # at a local maximum the limiter returns the cell value (first order)
    z = np.array([0.0, 1.0, 2.0, 3.0, 5.0, 3.0, 2.0, 1.0, 0.0, -1.0])[None, :]
    Lz = jo._muscl(z, 1, None, True)[0]
    Rz = jo._muscl(z, 1, None, False)[0]
    assert Lz[2] == 5.0  # left state at the face right of the peak cell (padded 4)
    assert Rz[1] == 5.0  # right state at the face left of it


def test_oracle_muscl_uniform_state_stationary(omech):
    nx, ny = 10, 8
    Y = np.tile(jo.stoich_Y(omech, 1.0)[:, None, None], (1, nx, ny))
    U0, a0 = jo.state_from_PTY(omech, np.full((1, nx, ny), 101325.0), np.full((1, nx, ny), 300.0), Y)
    bc = {k: "periodic" for k in BC2}
    for fc in FC.values():
        o = jo.Solver(omech, "2D", 1e-4, 1e-4, bc, 0.5, flux_config=fc)
        assert np.max(np.abs(o.flux_func(U0, a0, 1e-4, 1e-4, 1e-7))) == 0.0


# ---------------------------------------------------------------- GPU
def cuda(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


def _state2d(om, nx, ny, seed):
    rng = np.random.default_rng(seed)
    P = np.full((1, nx, ny), 101325.0)
    T = np.full((1, nx, ny), 300.0)
    Y = np.tile(jo.stoich_Y(om, 1.0)[:, None, None], (1, nx, ny))
    P[:, :4] = 30 * 101325.0
    T[:, :4] = 3000.0 * (1 + 0.05 * rng.uniform(-1, 1, (1, 4, ny)))
    U, aux = jo.state_from_PTY(om, P, T, Y)
    U[1] += U[0] * rng.uniform(-50.0, 50.0, (nx, ny))
    U[2] += U[0] * rng.uniform(-50.0, 50.0, (nx, ny))
    return U, jo.update_aux(om, U, aux)


def _state1d(om, nx, seed):
    rng = np.random.default_rng(seed)
    P = np.full((1, nx), 101325.0)
    T = np.full((1, nx), 300.0)
    Y = np.tile(jo.stoich_Y(om, 1.0)[:, None], (1, nx))
    P[:, :4] = 30 * 101325.0
    T[:, :4] = 3000.0
    U, aux = jo.state_from_PTY(om, P, T, Y)
    U[1] += U[0] * rng.uniform(-50.0, 50.0, nx)
    return U, jo.update_aux(om, U, aux)


COMBOS = [("slip_wall", "zero_gradient", "slip_wall", "slip_wall"),
          ("periodic", "periodic", "periodic", "periodic"),
          ("pressure_outlet", "zero_gradient", "no_slip_wall", "pressure_outlet")]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64_strict", "fp64"])
@pytest.mark.parametrize("scheme", list(FC))
@pytest.mark.parametrize("combo", COMBOS)
def test_muscl_flux_2d_vs_oracle(omech, prec, scheme, combo):
    from janc_b200.solver import Solver
    bc = dict(zip(["left_boundary", "right_boundary", "bottom_boundary", "top_boundary"], combo))
    nx, ny = 37, 23
    U, aux = _state2d(omech, nx, ny, 5)
    theta = {"Pb": 101325.0 * 1.3}
    o = jo.Solver(omech, "2D", 1e-4, 2e-4, bc, 0.5, flux_config=FC[scheme])
    ref = o.flux_func(U, aux, 1e-4, 2e-4, 2e-8, theta)
    s = Solver(2, nx, ny, 1e-4, 2e-4, bc, precision=prec, flux_config=FC[scheme])
    r = host(s.flux_func(cuda(U), cuda(aux), 1e-4, 2e-4, 2e-8, theta))
    assert field_err(r, ref) < (1e-13 if prec == "fp64_strict" else 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64_strict", "fp64"])
@pytest.mark.parametrize("scheme", list(FC))
def test_muscl_steps_1d_vs_oracle(omech, prec, scheme):
    from janc_b200.solver import Solver
    nx = 300  # more than one 1D tile
    P = np.full((1, nx), 101325.0)
    T = np.full((1, nx), 300.0)
    Y = np.tile(jo.stoich_Y(omech, 1.0)[:, None], (1, nx))
    P[:, :8] = 30 * 101325.0
    T[:, :8] = 3000.0
    U0, aux0 = jo.state_from_PTY(omech, P, T, Y)
    bc = {"left_boundary": "slip_wall", "right_boundary": "pressure_outlet"}
    theta = {"Pb": 101325.0}
    o = jo.Solver(omech, "1D", 5e-5, None, bc, 0.5, flux_config=FC[scheme])
    U, aux, t = U0, aux0, 0.0
    for _ in range(5):
        U, aux, t, _ = o.advance_func(U, aux, t, theta)
    s = Solver(1, nx, dx=5e-5, boundary_config=bc, precision=prec, flux_config=FC[scheme])
    Ug, ag, _ = s.advance(cuda(U0), cuda(aux0), 5, cfl=0.5, theta=theta)
    tol = 1e-12 if prec == "fp64_strict" else 1e-10
    assert field_err(host(Ug), U) < tol
    assert field_err(host(ag), aux) < tol
    assert s.status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64_strict", "fp64"])
@pytest.mark.parametrize("scheme", list(FC))
def test_muscl_steps_2d_vs_oracle(omech, prec, scheme):
    from janc_b200.solver import Solver
    nx, ny = 37, 23
    U0, aux0 = _state2d(omech, nx, ny, 7)
    dx = 1.953125e-4
    o = jo.Solver(omech, "2D", dx, dx, BC2, 0.5, flux_config=FC[scheme])
    U, aux, t = U0, aux0, 0.0
    for _ in range(4):
        U, aux, t, _ = o.advance_func(U, aux, t)
    s = Solver(2, nx, ny, dx, dx, BC2, precision=prec, flux_config=FC[scheme])
    Ug, ag, _ = s.advance(cuda(U0), cuda(aux0), 4, cfl=0.5)
    tol = 1e-12 if prec == "fp64_strict" else 1e-10
    assert field_err(host(Ug), U) < tol
    assert field_err(host(ag), aux) < tol
    assert s.status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", list(FC))
@pytest.mark.parametrize("dim", [1, 2])
def test_muscl_mixed_close_to_fp64(omech, scheme, dim):
    from janc_b200.solver import Solver
    nx, ny = 40, 24
    U0, aux0 = _state2d(omech, nx, ny, 9) if dim == 2 else _state1d(omech, nx, 9)
    out = []
    for prec in ("fp64", "mixed"):
        if dim == 2:
            s = Solver(2, nx, ny, 1e-4, 1e-4, BC2, precision=prec, flux_config=FC[scheme])
        else:
            s = Solver(1, nx, dx=1e-4, boundary_config={"left_boundary": "slip_wall",
                                                        "right_boundary": "zero_gradient"},
                       precision=prec, flux_config=FC[scheme])
        U, a, _ = s.advance(cuda(U0), cuda(aux0), 3, cfl=0.5)
        out.append((host(U), host(a)))
        assert s.status() == 0
    assert field_err(out[1][0], out[0][0]) < 1e-4
    assert field_err(out[1][0][:1], out[0][0][:1]) < 1e-6
    assert field_err(out[1][1], out[0][1]) < 1e-6
