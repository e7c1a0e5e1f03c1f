"""Steger-Warming flux splitting (flux_splitting/SW.py) with WENO5-JS or
MUSCL on the split fluxes.

CPU: the oracle's split satisfies H+ + H- = F (the Euler flux) in every row
but the energy (the Steger-Warming form assumes E = p/(gamma-1) + rho|u|^2/2,
which NASA7 thermo does not give) and keeps a uniform gas at rest; these pin
the restatement without the reference.  The reference's 1D SW cannot be
called (its split_flux takes a third `metrics` argument flux_splitting does
not pass); the oracle and the kernels use the arithmetic it states with
J = 1.
GPU (through the C ABI): flux_func and RK steps against the oracle.
Tolerances: ``fp64_strict`` 1e-13 relative L1 per field for one flux and
1e-12 over steps; ``fp64`` 1e-12 and 1e-10; ``mixed`` 1e-4 per field and
1e-6 on the density against the fp64 build.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import janc_oracle as jo  # noqa: E402

FC = {r: {"solver_type": "flux_splitting", "interface_reconstruction": r, "split_method": "SW",
          "viscosity": "off"} for r in ("WENO5_JS", "MUSCL")}
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
    P[:, :8] = 30 * 101325.0
    T[:, :8] = 3000.0
    U, aux = jo.state_from_PTY(om, P, T, Y)
    U[1] += U[0] * rng.uniform(-50.0, 50.0, nx)
    return U, jo.update_aux(om, U, aux)


# ---------------------------------------------------------------- CPU
@pytest.mark.parametrize("dim", [1, 2])
def test_oracle_sw_sums_to_euler_flux(omech, dim):
    U, a = _state2d(omech, 12, 10, 1) if dim == 2 else _state1d(omech, 40, 1)
    nE = 3 if dim == 2 else 2
    for ixy in ((1, 2) if dim == 2 else (1,)):
        if dim == 2:
            Hp, Hm = jo.split_sw_2d(omech, ixy, U, a)
            rho, u, v, Y, p, c = jo.U_to_prim(omech, U, a)
            vn = u if ixy == 1 else v
            F = [rho * vn, rho * u * vn + (p if ixy == 1 else 0), rho * v * vn + (p if ixy == 2 else 0),
                 vn * (U[3:4] + p), rho * vn * Y]
        else:
            Hp, Hm = jo.split_sw_1d(omech, U, a)
            rho, u, Y, p, c = jo.U_to_prim(omech, U, a)
            F = [rho * u, rho * u * u + p, u * (U[2:3] + p), rho * u * Y]
        F = np.concatenate(F, axis=0)
        S = Hp + Hm
        rows = [i for i in range(F.shape[0]) if i != nE]
        scale = np.max(np.abs(F[rows]), axis=(1,) if dim == 1 else (1, 2), keepdims=True) + 1e-300
        assert np.max(np.abs(S[rows] - F[rows]) / scale) < 1e-11
        assert np.max(np.abs(S[nE] - F[nE])) > 1e-6 * np.max(np.abs(F[nE]))  # not a perfect gas
        assert np.all(Hp[0] >= 0) and np.all(Hm[0] <= 0)  # mass: upwind halves


def test_oracle_sw_uniform_state_stationary(omech):
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


COMBOS = [("slip_wall", "zero_gradient", "slip_wall", "slip_wall"),
          ("periodic", "periodic", "periodic", "periodic"),
          ("pressure_outlet", "zero_gradient", "no_slip_wall", "pressure_outlet")]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64_strict", "fp64"])
@pytest.mark.parametrize("recon", list(FC))
@pytest.mark.parametrize("combo", COMBOS)
def test_sw_flux_2d_vs_oracle(omech, prec, recon, combo):
    from janc_b200.solver import Solver
    bc = dict(zip(["left_boundary", "right_boundary", "bottom_boundary", "top_boundary"], combo))
    nx, ny = 37, 23
    U, aux = _state2d(omech, nx, ny, 5)
    theta = {"Pb": 101325.0 * 1.3}
    o = jo.Solver(omech, "2D", 1e-4, 2e-4, bc, 0.5, flux_config=FC[recon])
    ref = o.flux_func(U, aux, 1e-4, 2e-4, 2e-8, theta)
    s = Solver(2, nx, ny, 1e-4, 2e-4, bc, precision=prec, flux_config=FC[recon])
    r = host(s.flux_func(cuda(U), cuda(aux), 1e-4, 2e-4, 2e-8, theta))
    assert field_err(r, ref) < (1e-13 if prec == "fp64_strict" else 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64_strict", "fp64"])
@pytest.mark.parametrize("recon", list(FC))
def test_sw_steps_1d_vs_oracle(omech, prec, recon):
    from janc_b200.solver import Solver
    nx = 300
    U0, aux0 = _state1d(omech, nx, 3)
    bc = {"left_boundary": "slip_wall", "right_boundary": "pressure_outlet"}
    theta = {"Pb": 101325.0}
    o = jo.Solver(omech, "1D", 5e-5, None, bc, 0.5, flux_config=FC[recon])
    U, aux, t = U0, aux0, 0.0
    for _ in range(5):
        U, aux, t, _ = o.advance_func(U, aux, t, theta)
    s = Solver(1, nx, dx=5e-5, boundary_config=bc, precision=prec, flux_config=FC[recon])
    Ug, ag, _ = s.advance(cuda(U0), cuda(aux0), 5, cfl=0.5, theta=theta)
    tol = 1e-12 if prec == "fp64_strict" else 1e-10
    assert field_err(host(Ug), U) < tol
    assert field_err(host(ag), aux) < tol
    assert s.status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64_strict", "fp64"])
@pytest.mark.parametrize("recon", list(FC))
def test_sw_steps_2d_vs_oracle(omech, prec, recon):
    from janc_b200.solver import Solver
    nx, ny = 37, 23
    U0, aux0 = _state2d(omech, nx, ny, 7)
    dx = 1.953125e-4
    o = jo.Solver(omech, "2D", dx, dx, BC2, 0.5, flux_config=FC[recon])
    U, aux, t = U0, aux0, 0.0
    for _ in range(4):
        U, aux, t, _ = o.advance_func(U, aux, t)
    s = Solver(2, nx, ny, dx, dx, BC2, precision=prec, flux_config=FC[recon])
    Ug, ag, _ = s.advance(cuda(U0), cuda(aux0), 4, cfl=0.5)
    tol = 1e-12 if prec == "fp64_strict" else 1e-10
    assert field_err(host(Ug), U) < tol
    assert field_err(host(ag), aux) < tol
    assert s.status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [1, 2])
def test_sw_mixed_close_to_fp64(omech, dim):
    from janc_b200.solver import Solver
    nx, ny = 40, 24
    U0, aux0 = _state2d(omech, nx, ny, 9) if dim == 2 else _state1d(omech, nx, 9)
    out = []
    for prec in ("fp64", "mixed"):
        if dim == 2:
            s = Solver(2, nx, ny, 1e-4, 1e-4, BC2, precision=prec, flux_config=FC["WENO5_JS"])
        else:
            s = Solver(1, nx, dx=1e-4, boundary_config={"left_boundary": "slip_wall",
                                                        "right_boundary": "zero_gradient"},
                       precision=prec, flux_config=FC["WENO5_JS"])
        U, a, _ = s.advance(cuda(U0), cuda(aux0), 3, cfl=0.5)
        out.append((host(U), host(a)))
        assert s.status() == 0
    assert field_err(out[1][0], out[0][0]) < 1e-4
    assert field_err(out[1][0][:1], out[0][0][:1]) < 1e-6
    assert field_err(out[1][1], out[0][1]) < 1e-6
