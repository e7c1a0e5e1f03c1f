"""Boundary conditions given as functions (boundary/boundary.py:16-21,
37-42, 58-63, 79-84): the function receives the 3 boundary-adjacent layers
of U and aux (``padded[:, 3:6, 3:-3]`` left, ``[:, -6:-3, 3:-3]`` right,
``[:, 3:-3, 3:6]`` bottom, ``[:, 3:-3, -6:-3]`` top; 1D without the second
index) and theta, and returns the 3 ghost layers in padded order.  The
library packs the layers and calls back before each flux evaluation
(``jb_set_ghost_cells``); the kernels read the ghost layers as they read
any ghost state.

GPU: flux_func and RK steps against the oracle, which calls the same
functions on NumPy arrays, in 2D (functions on all four sides or mixed with
named sides; LF, HLLC, viscous: the padded corners keep the periodic wrap)
and 1D.  Tolerances: ``fp64_strict`` 1e-13 relative L1
per field for one flux and 1e-12 over steps; ``fp64`` 1e-12 and 1e-10;
``mixed`` 1e-4 per field and 1e-6 on the density against ``fp64``.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import janc_oracle as jo  # noqa: E402


def _flip(a, axis=1):
    if isinstance(a, np.ndarray):
        return np.flip(a, axis=axis)
    return a.flip(axis)


def _like(a, v):
    """v (a NumPy array) as an array of a's kind and device."""
    return torch.as_tensor(v, device=a.device) if isinstance(a, torch.Tensor) else v


def make_inflow(U_in, aux_in):
    """Left: a fixed inflow state in all three ghost columns."""
    def left(U, aux, theta=None):
        shape = (1,) * (U.ndim - 1)
        Ug = U * 0 + _like(U, U_in.reshape((-1,) + shape))
        ag = aux * 0 + _like(aux, aux_in.reshape((-1,) + shape))
        return Ug, ag
    return left


def reflect(U, aux, theta=None):
    """Right: mirror the three columns (ghost l = column nx-1-l) with the
    x momentum negated -- a reflecting wall."""
    Ug = _flip(U) * 1.0
    Ug[1] = -Ug[1]
    return Ug, _flip(aux) * 1.0


def make_inflow_y(U_in, aux_in):
    """Bottom: the inflow state (momentum along y) in all three ghost rows."""
    def bottom(U, aux, theta=None):
        Ug = U * 0 + _like(U, U_in.reshape(-1, 1, 1))
        ag = aux * 0 + _like(aux, aux_in.reshape(-1, 1, 1))
        return Ug, ag
    return bottom


def reflect_y(U, aux, theta=None):
    """Bottom or top: mirror the three rows with the y momentum negated."""
    Ug = _flip(U, 2) * 1.0
    Ug[2] = -Ug[2]
    return Ug, _flip(aux, 2) * 1.0


def field_err(a, b):
    errs = []
    for i in range(a.shape[0]):
        den = np.sum(np.abs(b[i]))
        if den > 1e-30:
            errs.append(np.sum(np.abs(a[i] - b[i])) / den)
    return max(errs)


@pytest.fixture(scope="module")
def omech():
    from janc_b200.mechanism import DEFAULT_MECHANISM
    return jo.load_mechanism(DEFAULT_MECHANISM)


def _case(om, dim, seed=3):
    """A state with a hot, compressed layer at the right wall and an inflow
    state (3 atm, 600 K, 400 m/s along x) for the left boundary function."""
    rng = np.random.default_rng(seed)
    shape = (1, 40, 24) if dim == 2 else (1, 300)
    P = np.full(shape, 101325.0)
    T = np.full(shape, 300.0)
    Y = np.tile(jo.stoich_Y(om, 1.0).reshape((-1,) + (1,) * (len(shape) - 1)), (1,) + shape[1:])
    P[:, -6:] = 20 * 101325.0
    T[:, -6:] = 2500.0
    U, aux = jo.state_from_PTY(om, P, T, Y)
    U[1] += U[0] * rng.uniform(-40.0, 40.0, shape[1:])
    aux = jo.update_aux(om, U, aux)
    one = np.ones((1, 1))
    vel = [400.0 * one] + ([0.0 * one] if dim == 2 else [])
    Ui, ai = jo.state_from_PTY(om, 3 * 101325.0 * one, 600.0 * one, jo.stoich_Y(om, 1.0)[:, None], vel=vel)
    return U, aux, Ui[:, 0], ai[:, 0]


def _inflow_y(om):
    one = np.ones((1, 1))
    Ui, ai = jo.state_from_PTY(om, 2 * 101325.0 * one, 500.0 * one, jo.stoich_Y(om, 1.0)[:, None],
                               vel=[0.0 * one, 150.0 * one])
    return Ui[:, 0], ai[:, 0]


CASES = {"lf": None,
         "hllc": {"solver_type": "godunov", "interface_reconstruction": "WENO5_JS", "riemann_solver": "HLLC",
                  "viscosity": "off"},
         "visc": {"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS", "split_method": "LF",
                  "viscosity": "on"}}
TC = {"viscosity_model": "Sutherland", "thermal_conductivity_model": "Prandtl number", "Pr": 0.72,
      "species_diffusivity_model": "Lewis number", "Le": 1.0}


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64_strict", "fp64"])
@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("dim", [1, 2])
def test_boundary_functions_vs_oracle(omech, prec, case, dim):
    from janc_b200.solver import Solver
    if dim == 1 and case == "hllc":
        pytest.skip("covered in 2D")
    U0, a0, Ui, ai = _case(omech, dim)
    left = make_inflow(Ui, ai)
    keys = ["left_boundary", "right_boundary", "bottom_boundary", "top_boundary"][: 2 * dim]
    if dim == 2 and case == "lf":  # functions on all four sides
        Uy, ay = _inflow_y(omech)
        sides = [left, reflect, make_inflow_y(Uy, ay), reflect_y]
    elif dim == 2 and case == "visc":  # mixed with a named side
        sides = [left, reflect, reflect_y, "slip_wall"]
    else:
        sides = [left, reflect, "slip_wall", "slip_wall"]
    bc = dict(zip(keys, sides))
    dx = 5e-5
    fc, tc = CASES[case], (TC if case == "visc" else None)
    o = jo.Solver(omech, "2D" if dim == 2 else "1D", dx, dx if dim == 2 else None, bc, 0.4, flux_config=fc,
                  transport_config=tc)
    if dim == 2:
        s = Solver(2, U0.shape[1], U0.shape[2], dx, dx, bc, precision=prec, flux_config=fc, transport_config=tc)
    else:
        s = Solver(1, U0.shape[1], dx=dx, boundary_config=bc, precision=prec, flux_config=fc, transport_config=tc)
    ref = o.flux_func(U0, a0, dx, dx if dim == 2 else None, 1e-8)
    cu = lambda x: torch.as_tensor(np.ascontiguousarray(x), device="cuda")  # noqa: E731
    r = s.flux_func(cu(U0), cu(a0), dx, dx if dim == 2 else None, 1e-8).cpu().numpy()
    assert field_err(r, ref) < (1e-13 if prec == "fp64_strict" else 1e-12)
    U, aux, t = U0, a0, 0.0
    for _ in range(3):
        U, aux, t, _ = o.advance_func(U, aux, t)
    Ug, ag, _ = s.advance(cu(U0), cu(a0), 3, cfl=0.4)
    tol = 1e-12 if prec == "fp64_strict" else 1e-10
    assert np.all(np.isfinite(U))
    assert field_err(Ug.cpu().numpy(), U) < tol and field_err(ag.cpu().numpy(), aux) < tol
    assert s.status() == 0 and s._exchange.calls == 1 + 9


@pytest.mark.gpu
def test_boundary_function_errors_propagate(omech):
    from janc_b200.solver import Solver
    U0, a0, Ui, ai = _case(omech, 1)

    def broken(U, aux, theta=None):
        raise ValueError("user boundary failed")
    s = Solver(1, U0.shape[1], dx=5e-5, boundary_config={"left_boundary": broken, "right_boundary": reflect})
    with pytest.raises(Exception, match="user boundary failed"):
        s.flux_func(torch.as_tensor(U0, device="cuda"), torch.as_tensor(a0, device="cuda"), 5e-5, None, 1e-8)


def test_set_boundary_takes_functions_on_every_side():
    from janc_b200.janc.boundary import boundary
    boundary.set_boundary({"left_boundary": reflect, "right_boundary": "slip_wall",
                           "bottom_boundary": reflect_y, "top_boundary": reflect_y}, "2D")
    with pytest.raises(KeyError):
        boundary.set_boundary({"left_boundary": "inflow", "right_boundary": "slip_wall",
                               "bottom_boundary": "slip_wall", "top_boundary": "slip_wall"}, "2D")
