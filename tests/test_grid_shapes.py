"""Grid shapes at the edges of the kernels' tilings: the smallest grids the
reference's pad allows (4 cells per axis; boundary_padding.py takes cells
n-4 .. n-2), sizes below and just above a tile or warp run (the mixed y
runs are 32 cells, the x sweep segments 16, the 2D tiles 15 x 16, the 1D
tiles 255), against the oracle for every flux path; smaller grids are
refused when the handle is created.

Tolerances: float64 paths 1e-10 relative L1 per field over the steps;
mixed (float32 LF / WENO) 1e-4 per field (the mixed-precision bar) and
1e-6 on the density.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from janc_b200.solver import Solver  # noqa: E402
from oracle import janc_oracle as jo  # noqa: E402

BC = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient",
      "bottom_boundary": "periodic", "top_boundary": "periodic"}
SHAPES = [(4, 4), (5, 4), (4, 7), (16, 31), (17, 33), (33, 4), (70, 65)]
PATHS = {
    "lf_fp64": ("fp64", None, None),
    "lf_mixed": ("mixed", None, None),
    "hllc": ("fp64", {"solver_type": "godunov", "interface_reconstruction": "WENO5_JS",
                      "riemann_solver": "HLLC", "viscosity": "off"}, None),
    "hllc_mixed": ("mixed", {"solver_type": "godunov", "interface_reconstruction": "WENO5_JS",
                             "riemann_solver": "HLLC", "viscosity": "off"}, None),
    "lf_viscous": ("fp64", {"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS",
                            "split_method": "LF", "viscosity": "on"},
                   {"viscosity_model": "Sutherland", "thermal_conductivity_model": "Prandtl number",
                    "Pr": 0.72, "species_diffusivity_model": "Lewis number", "Le": 1.0}),
}


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


def _state(om, nx, ny, seed):
    """Smooth fields (a few random Fourier modes), so that the oracle's own
    run stays finite on every path."""
    rng = np.random.default_rng(seed)
    x = (np.arange(nx)[:, None] + 0.5) / nx
    y = (np.arange(ny)[None, :] + 0.5) / ny

    def smooth():
        f = np.zeros((nx, ny))
        for _ in range(3):
            kx, ky = rng.integers(1, 3, 2)
            f += rng.uniform(-1, 1) * np.sin(2 * np.pi * (kx * x + rng.uniform())) * np.cos(
                2 * np.pi * (ky * y + rng.uniform()))
        return f / 3

    P = (101325.0 * (1 + 0.2 * smooth()))[None]
    T = (1000.0 + 400.0 * smooth())[None]
    Y = np.tile(jo.stoich_Y(om, 1.0)[:, None, None], (1, nx, ny))
    U, aux = jo.state_from_PTY(om, P, T, Y)
    U[1] += U[0] * 30.0 * smooth()
    U[2] += U[0] * 30.0 * smooth()
    return U, jo.update_aux(om, U, aux)


@pytest.mark.parametrize("path", list(PATHS))
@pytest.mark.parametrize("shape", SHAPES)
def test_2d_shapes_vs_oracle(omech, path, shape):
    prec, fc, tc = PATHS[path]
    nx, ny = shape
    U0, aux0 = _state(omech, nx, ny, nx * 100 + ny)
    dx = 5e-5
    o = jo.Solver(omech, "2D", dx, dx, BC, 0.2, flux_config=fc, transport_config=tc)
    U, aux, t = U0, aux0, 0.0
    for _ in range(2):
        U, aux, t, _ = o.advance_func(U, aux, t)
    assert np.isfinite(U).all()
    s = Solver(2, nx, ny, dx, dx, BC, precision=prec, flux_config=fc, transport_config=tc)
    Ug, ag, _ = s.advance(torch.as_tensor(U0, device="cuda"), torch.as_tensor(aux0, device="cuda"), 2, cfl=0.2)
    torch.cuda.synchronize()
    tol = 1e-4 if prec == "mixed" else 1e-10
    Ug = Ug.cpu().numpy()
    assert field_err(Ug, U) < tol
    assert field_err(ag.cpu().numpy(), aux) < tol
    assert field_err(Ug[:1], U[:1]) < (1e-6 if prec == "mixed" else 1e-10)


@pytest.mark.parametrize("path", ["lf_fp64", "lf_mixed", "hllc", "hllc_mixed"])
@pytest.mark.parametrize("nx", [4, 5, 254, 255, 256, 511])
def test_1d_shapes_vs_oracle(omech, path, nx):
    prec, fc, tc = PATHS[path]
    rng = np.random.default_rng(nx)
    x = (np.arange(nx) + 0.5) / nx
    P = (101325.0 * (1 + 0.2 * np.sin(2 * np.pi * (x + rng.uniform()))))[None]
    T = (1000.0 + 400.0 * np.sin(2 * np.pi * (2 * x + rng.uniform())))[None]
    Y = np.tile(jo.stoich_Y(omech, 1.0)[:, None], (1, nx))
    U0, aux0 = jo.state_from_PTY(omech, P, T, Y)
    bc = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"}
    o = jo.Solver(omech, "1D", 5e-5, None, bc, 0.2, flux_config=fc)
    U, aux, t = U0, aux0, 0.0
    for _ in range(2):
        U, aux, t, _ = o.advance_func(U, aux, t)
    assert np.isfinite(U).all()
    s = Solver(1, nx, dx=5e-5, boundary_config=bc, precision=prec, flux_config=fc)
    Ug, ag, _ = s.advance(torch.as_tensor(U0, device="cuda"), torch.as_tensor(aux0, device="cuda"), 2, cfl=0.2)
    torch.cuda.synchronize()
    tol = 1e-4 if prec == "mixed" else 1e-10
    Ug = Ug.cpu().numpy()
    assert field_err(Ug, U) < tol
    assert field_err(Ug[:1], U[:1]) < (1e-6 if prec == "mixed" else 1e-10)


@pytest.mark.parametrize("shape", [(3, 8), (8, 3), (1, 1)])
def test_grids_below_the_pad_are_refused(shape):
    """The reference cannot pad an axis shorter than 4 cells; the handle
    refuses it before any kernel could index a ghost outside the grid."""
    with pytest.raises(RuntimeError):
        Solver(2, shape[0], shape[1], 1e-4, 1e-4, BC)
    with pytest.raises(RuntimeError):
        Solver(1, 3, dx=1e-4, boundary_config={"left_boundary": "slip_wall", "right_boundary": "zero_gradient"})
