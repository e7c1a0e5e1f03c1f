"""The reference's functions on ghost-padded arrays, through the drop-in
modules: boundary_conditions_1D / _2D (boundary/boundary.py:120-132) return
the padded (U, aux) as the kernels see them, corners included, and
total_flux (solver_{1D,2D}/flux.py) takes padded arrays and uses their ghost
layers.  GPU, against the oracle: padding bit for bit in ``fp64_strict``
(every entry, corners included); total_flux within 1e-13 (strict) relative
L1 per field, for the LF, Godunov and viscous fluxes."""
import numpy as np
import pytest

from oracle import janc_oracle as jo

KEYS = ["left_boundary", "right_boundary", "bottom_boundary", "top_boundary"]
COMBOS = [("slip_wall", "zero_gradient", "no_slip_wall", "pressure_outlet"),
          ("periodic", "periodic", "slip_wall", "zero_gradient"),
          ("pressure_outlet", "no_slip_wall", "periodic", "periodic")]


def _state(om, dim, seed=2):
    rng = np.random.default_rng(seed)
    shape = (1, 20, 14) if dim == 2 else (1, 40)
    P = 101325.0 * (1 + 0.2 * rng.uniform(-1, 1, shape))
    T = 300.0 + 900.0 * rng.uniform(0, 1, shape)
    Y = np.tile(jo.stoich_Y(om, 1.0).reshape((-1,) + (1,) * (len(shape) - 1)), (1,) + shape[1:])
    U, aux = jo.state_from_PTY(om, P, T, Y)
    for k in range(1, dim + 1):
        U[k] += U[0] * rng.uniform(-60.0, 60.0, shape[1:])
    return U, jo.update_aux(om, U, aux)


def _configure(dim, bc, flux=None, transport=None):
    from janc_b200.janc import _state
    from janc_b200.janc.boundary import boundary
    from janc_b200.janc.solver_1D import flux as flux1
    from janc_b200.janc.solver_2D import flux as flux2
    _state.reset_solvers()
    _state.config["precision"] = "fp64_strict"
    boundary.set_boundary(bc, "2D" if dim == 2 else "1D")
    fc = flux or {"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS", "split_method": "LF",
                  "viscosity": "off"}
    (flux2 if dim == 2 else flux1).set_flux_solver(fc, transport)


@pytest.mark.gpu
@pytest.mark.parametrize("combo", COMBOS)
@pytest.mark.parametrize("dim", [1, 2])
def test_boundary_conditions_bitwise(combo, dim):
    from janc_b200.janc.boundary import boundary
    from janc_b200.mechanism import DEFAULT_MECHANISM
    om = jo.load_mechanism(DEFAULT_MECHANISM)
    bc = dict(zip(KEYS[: 2 * dim], combo))
    _configure(dim, bc)
    U, aux = _state(om, dim)
    theta = {"Pb": 1.4 * 101325.0}
    Up, Ap = (boundary.boundary_conditions_2D if dim == 2 else boundary.boundary_conditions_1D)(U, aux, theta)
    Ur, Ar = jo.boundary_conditions(om, U, aux, bc, theta)
    np.testing.assert_array_equal(Up, Ur)
    np.testing.assert_array_equal(Ap, Ar)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["lf", "hllc", "visc"])
@pytest.mark.parametrize("dim", [1, 2])
def test_total_flux_of_padded_arrays(case, dim):
    from janc_b200.janc.solver_1D import flux as flux1
    from janc_b200.janc.solver_2D import flux as flux2
    from janc_b200.mechanism import DEFAULT_MECHANISM
    om = jo.load_mechanism(DEFAULT_MECHANISM)
    fc = {"lf": None,
          "hllc": {"solver_type": "godunov", "interface_reconstruction": "WENO5_JS", "riemann_solver": "HLLC",
                   "viscosity": "off"},
          "visc": {"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS", "split_method": "LF",
                   "viscosity": "on"}}[case]
    tc = {"viscosity_model": "Sutherland", "thermal_conductivity_model": "Prandtl number", "Pr": 0.72,
          "species_diffusivity_model": "Lewis number", "Le": 1.0} if case == "visc" else None
    bc = dict(zip(KEYS[: 2 * dim], COMBOS[0]))
    _configure(dim, bc, fc, tc)
    U, aux = _state(om, dim)
    Up, Ap = jo.boundary_conditions(om, U, aux, bc, {"Pb": 1.4 * 101325.0})
    dx = 3e-5
    o = jo.Solver(om, "2D" if dim == 2 else "1D", dx, dx if dim == 2 else None, bc, 0.4, flux_config=fc,
                  transport_config=tc)
    ref = o.padded_rhs(Up, Ap, dx, dx if dim == 2 else None, 1.0)
    got = flux2.total_flux(Up, Ap, dx, dx) if dim == 2 else flux1.total_flux(Up, Ap, dx)
    assert got.shape == ref.shape
    err = max(np.sum(np.abs(got[i] - ref[i])) / np.sum(np.abs(ref[i])) for i in range(ref.shape[0])
              if np.sum(np.abs(ref[i])) > 1e-30)
    assert err < 1e-13


@pytest.mark.gpu
def test_prim_to_U_inverts_U_to_prim():
    """aux_func.prim_to_U(U_to_prim(U)) returns U and the state's (gamma, T)
    (the reference's own prim_to_U cannot run: its kinetic term calls rho)."""
    from janc_b200.janc.solver_2D import aux_func
    from janc_b200.mechanism import DEFAULT_MECHANISM
    om = jo.load_mechanism(DEFAULT_MECHANISM)
    _configure(2, dict(zip(KEYS, COMBOS[0])))
    U, aux = _state(om, 2)
    rho, u, v, Y, p, a = aux_func.U_to_prim(U, aux)
    U2, aux2 = aux_func.prim_to_U(np.concatenate([rho, u, v, p, Y], axis=0))
    for i in range(U.shape[0]):
        assert np.max(np.abs(U2[i] - U[i])) <= 1e-12 * np.max(np.abs(U[i])) + 1e-300
    assert np.max(np.abs(aux2[1] - aux[1]) / aux[1]) < 1e-13
    assert np.max(np.abs(aux2[0] - aux[0]) / aux[0]) < 1e-13
    g, T = aux_func.aux_to_thermo(U, aux)
    assert np.array_equal(g, aux[0:1]) and np.array_equal(T, aux[1:2])
    aux_func.set_source_terms(None)
    assert np.all(aux_func.source_terms(U, aux) == 0)
    aux_func.set_source_terms({"self_defined_source_terms": lambda U, a, th: 2 * U})
    assert np.array_equal(aux_func.source_terms(U, aux), 2 * U)
    aux_func.set_source_terms(None)


@pytest.mark.gpu
def test_get_thermo_properties_bitwise():
    """thermo_model.get_thermo_properties(T): per-species cp, dcp, h across
    both NASA7 ranges (the 1000 K switch included), bit for bit in strict."""
    from janc_b200.janc.model import thermo_model
    from janc_b200.mechanism import DEFAULT_MECHANISM
    om = jo.load_mechanism(DEFAULT_MECHANISM)
    _configure(2, dict(zip(KEYS, COMBOS[0])))
    T = np.concatenate([np.linspace(250.0, 3500.0, 61), [999.999, 1000.0, 1000.001]]).reshape(8, 8)
    cp, dcp, h = thermo_model.get_thermo_properties(T)
    rcp, rdcp, rh = jo.get_thermo_properties(om, T)
    np.testing.assert_array_equal(cp, rcp)
    np.testing.assert_array_equal(dcp, rdcp)
    np.testing.assert_array_equal(h, rh)
