"""Godunov path (solver_{1D,2D}/flux.py godunov_flux): WENO5-JS on the
primitives with the HLLC or AUSMPW+ Riemann solver.

CPU: the flux_config validation of set_flux_solver, and the oracle's
Riemann fluxes against identities that pin them without the reference
(consistency F(q, q) = Euler flux, a uniform gas stays at rest).
GPU (through the C ABI): flux_func and RK steps against the oracle.
Tolerances: ``fp64_strict`` 1e-13 relative L1 per field for one flux
evaluation and 1e-12 over steps; ``fp64`` 1e-12 and 1e-10; ``mixed``
(float32 reconstruction) 1e-4 per field and 1e-6 on the density.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import janc_oracle as jo  # noqa: E402

GOD = {s: {"solver_type": "godunov", "interface_reconstruction": "WENO5_JS", "riemann_solver": s,
           "viscosity": "off"} for s in ("HLLC", "AUSMPW_plus")}
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
def test_flux_config_validation():
    from janc_b200.solver import flux_scheme
    assert flux_scheme(None) == "LF"
    assert flux_scheme(GOD["HLLC"]) == "HLLC"
    assert flux_scheme(GOD["AUSMPW_plus"]) == "AUSMPW_plus"
    assert flux_scheme({"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS",
                        "split_method": "LF", "viscosity": "off"}) == "LF"
    with pytest.raises(KeyError, match="godunov"):
        flux_scheme({"solver_type": "spectral"})
    with pytest.raises(KeyError):
        flux_scheme({"solver_type": "godunov", "interface_reconstruction": "WENO5_JS", "riemann_solver": "Roe"})
    assert flux_scheme({"solver_type": "godunov", "interface_reconstruction": "MUSCL",
                        "riemann_solver": "HLLC"}) == "HLLC"
    with pytest.raises(KeyError):
        flux_scheme({"solver_type": "godunov", "interface_reconstruction": "WENO7", "riemann_solver": "HLLC"})
    assert flux_scheme({"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS",
                        "split_method": "SW"}) == "SW"
    with pytest.raises(KeyError):
        flux_scheme({"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS",
                     "split_method": "VanLeer"})


def _random_w(om, dim, n, rng):
    rho = rng.uniform(0.2, 3.0, (1, n))
    vel = rng.uniform(-900.0, 900.0, (dim, n))
    p = rng.uniform(2e4, 3e6, (1, n))
    Y = rng.dirichlet(np.ones(9), n).T[:8]
    return np.concatenate([rho, vel, p, Y], axis=0)


@pytest.mark.parametrize("rs", ["HLLC", "AUSMPW_plus"])
@pytest.mark.parametrize("dim,n", [(1, 1), (2, 1), (2, 2)])
def test_oracle_riemann_consistency(omech, rs, dim, n):
    """F(q, q) is the Euler flux of q in the face's normal direction."""
    rng = np.random.default_rng(11)
    w = _random_w(omech, dim, 200, rng)
    F = jo.RIEMANN[rs](omech, w, w, dim, n)
    rho, vel, p, Y = w[0:1], w[1:1 + dim], w[1 + dim:2 + dim], w[2 + dim:]
    gamma, h = jo._face_thermo(omech, rho, p, Y)
    un = vel[n - 1:n]
    E = rho * h - p + 0.5 * rho * np.sum(vel ** 2, axis=0, keepdims=True)
    mom = [rho * un * vel[k:k + 1] + (p if k == n - 1 else 0.0) for k in range(dim)]
    ref = np.concatenate([rho * un] + mom + [un * (E + p), rho * un * Y], axis=0)
    assert np.max(np.abs(F - ref) / (np.abs(ref) + 1e-12 * np.max(np.abs(ref), axis=1, keepdims=True))) < 1e-11


@pytest.mark.parametrize("rs", ["HLLC", "AUSMPW_plus"])
def test_oracle_uniform_state_stationary(omech, rs):
    nx, ny = 10, 8
    Y = np.tile(jo.stoich_Y(omech, 1.0)[:, None, None], (1, nx, ny))
    U0, a0 = jo.state_from_PTY(omech, np.full((1, nx, ny), 101325.0), np.full((1, nx, ny), 300.0), Y)
    bc = {k: "periodic" for k in BC2}
    o = jo.Solver(omech, "2D", 1e-4, 1e-4, bc, 0.5, flux_config=GOD[rs])
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
    U[1] += U[0] * rng.uniform(-50.0, 50.0, (nx, ny))  # a velocity field through every face
    U[2] += U[0] * rng.uniform(-50.0, 50.0, (nx, ny))
    aux = jo.update_aux(om, U, aux)
    return U, aux


COMBOS = [("slip_wall", "zero_gradient", "slip_wall", "slip_wall"),
          ("periodic", "periodic", "periodic", "periodic"),
          ("pressure_outlet", "zero_gradient", "no_slip_wall", "pressure_outlet")]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64_strict", "fp64"])
@pytest.mark.parametrize("rs", ["HLLC", "AUSMPW_plus"])
@pytest.mark.parametrize("combo", COMBOS)
def test_flux_2d_vs_oracle(omech, prec, rs, combo):
    from janc_b200.solver import Solver
    bc = dict(zip(["left_boundary", "right_boundary", "bottom_boundary", "top_boundary"], combo))
    nx, ny = 37, 23
    U, aux = _state2d(omech, nx, ny, 5)
    theta = {"Pb": 101325.0 * 1.3}
    o = jo.Solver(omech, "2D", 1e-4, 2e-4, bc, 0.5, flux_config=GOD[rs])
    ref = o.flux_func(U, aux, 1e-4, 2e-4, 2e-8, theta)
    s = Solver(2, nx, ny, 1e-4, 2e-4, bc, precision=prec, flux_config=GOD[rs])
    r = host(s.flux_func(cuda(U), cuda(aux), 1e-4, 2e-4, 2e-8, theta))
    assert field_err(r, ref) < (1e-13 if prec == "fp64_strict" else 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64_strict", "fp64"])
@pytest.mark.parametrize("rs", ["HLLC", "AUSMPW_plus"])
def test_steps_1d_vs_oracle(omech, prec, rs):
    from janc_b200.solver import Solver
    nx = 300  # more than one 255-cell tile
    P = np.full((1, nx), 101325.0)
    T = np.full((1, nx), 300.0)
    Y = np.tile(jo.stoich_Y(omech, 1.0)[:, None], (1, nx))
    P[:, :8] = 30 * 101325.0
    T[:, :8] = 3000.0
    U0, aux0 = jo.state_from_PTY(omech, P, T, Y)
    bc = {"left_boundary": "slip_wall", "right_boundary": "pressure_outlet"}
    theta = {"Pb": 101325.0}
    o = jo.Solver(omech, "1D", 5e-5, None, bc, 0.5, flux_config=GOD[rs])
    U, aux, t = U0, aux0, 0.0
    for _ in range(5):
        U, aux, t, _ = o.advance_func(U, aux, t, theta)
    s = Solver(1, nx, dx=5e-5, boundary_config=bc, precision=prec, flux_config=GOD[rs])
    Ug, ag, _ = s.advance(cuda(U0), cuda(aux0), 5, cfl=0.5, theta=theta)
    tol = 1e-12 if prec == "fp64_strict" else 1e-10
    assert field_err(host(Ug), U) < tol
    assert field_err(host(ag), aux) < tol
    assert s.status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64_strict", "fp64"])
@pytest.mark.parametrize("rs", ["HLLC", "AUSMPW_plus"])
def test_steps_2d_vs_oracle(omech, prec, rs):
    from janc_b200.solver import Solver
    nx, ny = 37, 23
    U0, aux0 = _state2d(omech, nx, ny, 7)
    dx = 1.953125e-4
    o = jo.Solver(omech, "2D", dx, dx, BC2, 0.5, flux_config=GOD[rs])
    U, aux, t = U0, aux0, 0.0
    for _ in range(4):
        U, aux, t, _ = o.advance_func(U, aux, t)
    s = Solver(2, nx, ny, dx, dx, BC2, precision=prec, flux_config=GOD[rs])
    Ug, ag, _ = s.advance(cuda(U0), cuda(aux0), 4, cfl=0.5)
    tol = 1e-12 if prec == "fp64_strict" else 1e-10
    assert field_err(host(Ug), U) < tol
    assert field_err(host(ag), aux) < tol
    assert s.status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("rs", ["HLLC", "AUSMPW_plus"])
def test_mixed_godunov_close_to_fp64(omech, rs):
    """The mixed build reconstructs the primitives in float32 (Riemann
    solver, RK and temperature solve in float64): within the mixed bar of
    the fp64 build after three steps."""
    from janc_b200.solver import Solver
    nx, ny = 40, 24
    U0, aux0 = _state2d(omech, nx, ny, 9)
    out = []
    for prec in ("fp64", "mixed"):
        s = Solver(2, nx, ny, 1e-4, 1e-4, BC2, precision=prec, flux_config=GOD[rs])
        U, a, _ = s.advance(cuda(U0), cuda(aux0), 3, cfl=0.5)
        out.append((host(U), host(a)))
        assert s.status() == 0
    assert field_err(out[1][0], out[0][0]) < 1e-4
    assert field_err(out[1][0][:1], out[0][0][:1]) < 1e-6
    assert field_err(out[1][1], out[0][1]) < 1e-6
