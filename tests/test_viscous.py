"""Laminar viscous fluxes (solver_{1D,2D}/flux.py viscous_flux_node /
viscous_flux, model/transport_model.py, CENTRAL6 derivatives and interfaces).

CPU: set_transport's parsing and errors; the oracle's CENTRAL6 stencils are
exact on polynomials of their order (pins the restatement without the
reference); a uniform gas has no viscous flux.
GPU (through the C ABI): flux_func with viscosity against the oracle for
each transport model (laminar and LES with the Vreman sub-grid viscosity)
and boundary set (padded corners included), and RK steps.  Tolerances: ``fp64_strict`` 1e-12 relative L1 per field (the
Sutherland law goes through pow), ``fp64`` 1e-11 per flux and 1e-10 over
steps, ``mixed`` 1e-4 per field and 1e-6 on the density.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import janc_oracle as jo  # noqa: E402

LF_VISC = {"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS", "split_method": "LF",
           "viscosity": "on"}
HLLC_VISC = {"solver_type": "godunov", "interface_reconstruction": "WENO5_JS", "riemann_solver": "HLLC",
             "viscosity": "on"}
TRANSPORT = {
    "sutherland_pr_le": {"viscosity_model": "Sutherland", "thermal_conductivity_model": "Prandtl number",
                         "Pr": 0.72, "species_diffusivity_model": "Lewis number", "Le": 1.0},
    "sutherland_sc": {"viscosity_model": "Sutherland", "reference_viscosity": 1.8e-5,
                      "thermal_conductivity_model": "Prandtl number", "Pr": 0.7,
                      "species_diffusivity_model": "Schmidt number", "Sc": 0.5},
    "constant_all": {"viscosity_model": "constant", "dynamic_viscosity": 2e-5,
                     "thermal_conductivity_model": "constant", "thermal_conductivity": 0.05,
                     "species_diffusivity_model": "constant", "species_diffusivity": 3e-5},
    "constant_mu_le": {"viscosity_model": "constant", "dynamic_viscosity": 1.5e-5,
                       "thermal_conductivity_model": "constant", "thermal_conductivity": 0.04,
                       "species_diffusivity_model": "Lewis number", "Le": 0.8},
    # LES with the Vreman sub-grid viscosity (model/LES/Verman.py)
    "les_pr_le": {"viscosity_model": "Sutherland", "thermal_conductivity_model": "Prandtl number", "Pr": 0.72,
                  "species_diffusivity_model": "Lewis number", "Le": 1.0, "turbulence_model": "LES",
                  "LES_model": "Verman", "Pr_t": 0.9, "Le_t": 1.1},
    "les_constant": {"viscosity_model": "constant", "dynamic_viscosity": 2e-5,
                     "thermal_conductivity_model": "constant", "thermal_conductivity": 0.05,
                     "species_diffusivity_model": "constant", "species_diffusivity": 3e-5,
                     "turbulence_model": "LES", "LES_model": "Verman", "Pr_t": 0.85, "Sc_t": 0.7},
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


# ---------------------------------------------------------------- CPU
def test_transport_config_parsing():
    from janc_b200.solver import transport_params
    t = transport_params(TRANSPORT["sutherland_sc"])
    assert (t.viscosity_model, t.conductivity_model, t.diffusivity_model) == (0, 0, 0)
    assert t.mu_ref == 1.8e-5 and t.T_ref == 273.15 and t.S == 110.4
    assert t.Pr == 0.7 and t.Le == 0.5 / 0.7
    t = transport_params(TRANSPORT["constant_all"])
    assert (t.viscosity_model, t.conductivity_model, t.diffusivity_model) == (1, 1, 1)
    assert (t.nu0, t.k0, t.D0) == (2e-5, 0.05, 3e-5)
    with pytest.raises(KeyError):
        transport_params({"viscosity_model": "power_law"})
    with pytest.raises(AssertionError):
        transport_params({"viscosity_model": "Sutherland", "thermal_conductivity_model": "Prandtl number"})
    with pytest.raises(AssertionError):  # LES needs LES_model, Pr_t and Le_t / Sc_t
        transport_params(dict(TRANSPORT["sutherland_pr_le"], turbulence_model="LES"))
    les = dict(TRANSPORT["sutherland_pr_le"], turbulence_model="LES", LES_model="Verman", Pr_t=0.9, Sc_t=0.7)
    t = transport_params(les)
    assert t.turbulence_model == 1 and t.Pr_t == 0.9 and t.Le_t == 0.7 / 0.9
    with pytest.raises(KeyError, match="Verman_1D"):
        transport_params(les, dim=1)
    with pytest.raises(KeyError, match="WALE_2D"):
        transport_params(dict(les, LES_model="WALE"))
    with pytest.raises(KeyError):
        transport_params(dict(les, turbulence_model="RANS"))
    # the oracle parses the same way
    tr = jo.Transport(TRANSPORT["sutherland_sc"])
    assert tr.Le == 0.5 / 0.7 and tr.D_type == "Lewis number"


def test_oracle_vreman_pure_strain_closed_form():
    """u = a x, v = -a y: B = dx^2 dy^2 a^4, a_ij a_ij = 2 a^2, so
    mu_t = 0.07 rho dx dy |a| / sqrt(2); simple shear gives mu_t = 0 in the
    2D form."""
    tr = jo.Transport(TRANSPORT["les_pr_le"])
    rho = np.array([[1.3, 0.4]])
    a = np.array([[250.0, -70.0]])
    z = np.zeros_like(a)
    mu, mu_t = tr.mu_total(rho, np.full_like(rho, 900.0), 2e-5, 3e-5, a, z, z, -a)
    ref = 0.07 * rho * 2e-5 * 3e-5 * np.abs(a) / np.sqrt(2.0)
    assert np.allclose(mu_t, ref, rtol=1e-13)
    assert np.allclose(mu, tr.mu(rho, np.full_like(rho, 900.0)) + ref, rtol=1e-13)
    _, mu_t = tr.mu_total(rho, np.full_like(rho, 900.0), 2e-5, 3e-5, z, a, z, z)
    assert np.all(mu_t == 0.0)
    _, mu_t = tr.mu_total(rho, np.full_like(rho, 900.0), 2e-5, 3e-5, z, z, z, z)
    assert np.all(mu_t == 0.0)  # a_sum = 0: the reference's where() gives 0


def test_central6_stencils_exact_on_polynomials():
    """d_dx: sixth-order central inside (exact to degree 6), the one-sided
    forms exact to degree 1, 2 and 4; interface: exact to degree 5."""
    x = np.arange(20, dtype=np.float64) * 0.1
    for deg, where in ((6, slice(3, -3)), (4, [2, -3]), (2, [1, -2]), (1, [0, -1])):
        c = np.arange(1, deg + 2, dtype=np.float64)
        f = np.polyval(c, x)[None, :]
        d = jo._d_axis(f, 0.1, 1)[0]
        exact = np.polyval(np.polyder(c), x)
        assert np.max(np.abs(d[where] - exact[where])) < 1e-8 * np.max(np.abs(exact)), deg
    c = np.arange(1, 7, dtype=np.float64)
    xp = np.arange(26, dtype=np.float64) * 0.1
    fv = np.polyval(c, xp)[None, :, None] * np.ones((1, 1, 8))
    fi = jo._central6_interface(fv, 1, 2)[0, :, 0]
    mid = (xp[2:-3] + xp[3:-2]) / 2
    assert np.max(np.abs(fi - np.polyval(c, mid))) < 1e-9 * np.max(np.abs(fi))


def test_oracle_uniform_gas_has_no_viscous_flux(omech):
    nx, ny = 10, 8
    Y = np.tile(jo.stoich_Y(omech, 1.0)[:, None, None], (1, nx, ny))
    U0, a0 = jo.state_from_PTY(omech, np.full((1, nx, ny), 101325.0), np.full((1, nx, ny), 300.0), Y)
    bc = {k: "periodic" for k in ("left_boundary", "right_boundary", "bottom_boundary", "top_boundary")}
    Up, Ap = jo.boundary_conditions(omech, U0, a0, bc)
    v = jo.viscous_flux(omech, jo.Transport(TRANSPORT["sutherland_pr_le"]), Up, Ap, 1e-4, 1e-4)
    # the stencils sum to zero only up to rounding on a constant field
    assert np.max(np.abs(v)) <= 1e-12 * np.max(np.abs(U0)) / 1e-4


# ---------------------------------------------------------------- GPU
def cuda(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


def _state2d(om, nx, ny, seed):
    rng = np.random.default_rng(seed)
    P = np.full((1, nx, ny), 101325.0) * (1 + 0.1 * rng.uniform(-1, 1, (1, nx, ny)))
    T = 300.0 + 1500.0 * rng.uniform(0, 1, (1, nx, ny))
    Y = np.tile(jo.stoich_Y(om, 1.0)[:, None, None], (1, nx, ny))
    Y[:5] *= 1 + 0.2 * rng.uniform(-1, 1, (5, nx, ny))
    U, aux = jo.state_from_PTY(om, P, T, Y)
    U[1] += U[0] * rng.uniform(-80.0, 80.0, (nx, ny))
    U[2] += U[0] * rng.uniform(-80.0, 80.0, (nx, ny))
    return U, jo.update_aux(om, U, aux)


COMBOS = [("periodic", "periodic", "periodic", "periodic"),
          ("slip_wall", "zero_gradient", "no_slip_wall", "slip_wall"),
          ("pressure_outlet", "zero_gradient", "slip_wall", "pressure_outlet")]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64_strict", "fp64"])
@pytest.mark.parametrize("tkey", list(TRANSPORT))
@pytest.mark.parametrize("combo", COMBOS)
def test_viscous_flux_2d_vs_oracle(omech, prec, tkey, combo):
    from janc_b200.solver import Solver
    bc = dict(zip(["left_boundary", "right_boundary", "bottom_boundary", "top_boundary"], combo))
    nx, ny = 37, 23
    U, aux = _state2d(omech, nx, ny, 3)
    dx, dy = 2e-5, 3e-5
    theta = {"Pb": 101325.0}
    o = jo.Solver(omech, "2D", dx, dy, bc, 0.5, flux_config=LF_VISC, transport_config=TRANSPORT[tkey])
    ref = o.flux_func(U, aux, dx, dy, 1e-9, theta)
    s = Solver(2, nx, ny, dx, dy, bc, precision=prec, flux_config=LF_VISC, transport_config=TRANSPORT[tkey])
    r = host(s.flux_func(cuda(U), cuda(aux), dx, dy, 1e-9, theta))
    assert field_err(r, ref) < (1e-12 if prec == "fp64_strict" else 1e-11)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64_strict", "fp64", "mixed"])
@pytest.mark.parametrize("tkey", ["sutherland_pr_le", "les_pr_le"])
def test_viscous_godunov_steps_2d_vs_oracle(omech, prec, tkey):
    """(``les_constant`` is left to the flux comparison: the reference's
    constant-diffusivity turbulent term multiplies by cp_k,
    transport_model.py:153-155, which makes D large enough that the oracle's
    own steps go non-finite at these sizes.)"""
    from janc_b200.solver import Solver
    nx, ny = 37, 23
    U0, aux0 = _state2d(omech, nx, ny, 4)
    dx = 2e-5
    bc = dict(zip(["left_boundary", "right_boundary", "bottom_boundary", "top_boundary"], COMBOS[1]))
    tc = TRANSPORT[tkey]
    o = jo.Solver(omech, "2D", dx, dx, bc, 0.3, flux_config=HLLC_VISC, transport_config=tc)
    U, aux, t = U0, aux0, 0.0
    for _ in range(3):
        U, aux, t, _ = o.advance_func(U, aux, t)
    s = Solver(2, nx, ny, dx, dx, bc, precision=prec, flux_config=HLLC_VISC, transport_config=tc)
    Ug, ag, _ = s.advance(cuda(U0), cuda(aux0), 3, cfl=0.3)
    tol = {"fp64_strict": 1e-11, "fp64": 1e-10, "mixed": 1e-4}[prec]
    Ug = host(Ug)
    assert field_err(Ug, U) < tol
    assert field_err(host(ag), aux) < tol
    assert field_err(Ug[:1], U[:1]) < (1e-6 if prec == "mixed" else tol)
    assert s.status() == 0


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64_strict", "fp64", "mixed"])
@pytest.mark.parametrize("tkey", ["sutherland_pr_le", "constant_all"])
def test_viscous_steps_1d_vs_oracle(omech, prec, tkey):
    from janc_b200.solver import Solver
    nx = 300
    rng = np.random.default_rng(8)
    P = np.full((1, nx), 101325.0)
    T = 300.0 + 1200.0 * rng.uniform(0, 1, (1, nx))
    Y = np.tile(jo.stoich_Y(omech, 1.0)[:, None], (1, nx))
    U0, aux0 = jo.state_from_PTY(omech, P, T, Y)
    U0[1] += U0[0] * rng.uniform(-50.0, 50.0, nx)
    aux0 = jo.update_aux(omech, U0, aux0)
    bc = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"}
    fc = {"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS", "split_method": "LF",
          "viscosity": "on"}
    o = jo.Solver(omech, "1D", 2e-5, None, bc, 0.3, flux_config=fc, transport_config=TRANSPORT[tkey])
    U, aux, t = U0, aux0, 0.0
    for _ in range(4):
        U, aux, t, _ = o.advance_func(U, aux, t)
    s = Solver(1, nx, dx=2e-5, boundary_config=bc, precision=prec, flux_config=fc,
               transport_config=TRANSPORT[tkey])
    Ug, ag, _ = s.advance(cuda(U0), cuda(aux0), 4, cfl=0.3)
    tol = {"fp64_strict": 1e-11, "fp64": 1e-10, "mixed": 1e-5}[prec]
    assert field_err(host(Ug), U) < tol
    assert s.status() == 0
