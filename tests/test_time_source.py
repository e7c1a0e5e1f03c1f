"""The step's callers beyond the fused TVD_RK3 path (simulation/set_simulator.py
set_rhs / set_advance_func, simulation/time_step/RK2.py): Heun's RK2 and a
user source term (``source_config['self_defined_source_terms']``, added to
the flux for flux splitting, a second time-stepped pass for Godunov), each
composed from the native flux_func / update_aux / reaction_source_terms as
the reference composes them.

CPU: configuration errors.  GPU: Simulator.advance_func against the oracle's
composition (``fp64_strict``, 1e-12 relative L1 per field over 4 steps).
"""
import numpy as np
import pytest

from oracle import janc_oracle as jo

KEYS2 = ["left_boundary", "right_boundary", "bottom_boundary", "top_boundary"]
G = 9.81e4  # a body force strong enough to show within a few steps


def _cfg(dim, scheme="TVD_RK3", flux=None, source=None, detailed=True):
    from janc_b200.mechanism import DEFAULT_MECHANISM as MECH
    bc = dict(zip(KEYS2, ["slip_wall", "zero_gradient", "slip_wall", "slip_wall"]))
    cfg = {"dimension": dim, "grid_config": {"dx": 1e-4, "dy": 1e-4} if dim == "2D" else {"dx": 5e-5},
           "thermo_config": {"thermo_model": "nasa7", "mechanism_directory": MECH},
           "reaction_config": {"is_detailed_chemistry": detailed, "mechanism_directory": MECH},
           "flux_config": flux or {"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS",
                                   "split_method": "LF", "viscosity": "off"},
           "boundary_config": bc if dim == "2D" else {k: bc[k] for k in KEYS2[:2]},
           "time_config": {"temporal_evolution_scheme": scheme, "t_end": 1.0, "CFL": 0.4},
           "precision": "fp64_strict"}
    if source is not None:
        cfg["source_config"] = {"self_defined_source_terms": source}
    return cfg


def gravity(U, aux, dt, theta=None):
    """dt * (0, 0, -rho g, 0, -rho v g, 0 ...) in 2D: a body force along -y."""
    S = np.zeros_like(U)
    S[2] = -U[0] * G
    S[3] = -U[2] * G
    return dt * S


def test_config_errors():
    from janc_b200.janc.simulation.set_simulator import Simulator
    with pytest.raises(KeyError):
        Simulator(_cfg("2D", scheme="RK4"))
    with pytest.raises(NotImplementedError):
        Simulator(_cfg("2D", detailed=False))


def _state(om, dim):
    rng = np.random.default_rng(3)
    if dim == "2D":
        nx, ny = 40, 24
        shape = (1, nx, ny)
    else:
        nx, shape = 300, (1, 300)
    P = np.full(shape, 101325.0)
    T = np.full(shape, 300.0)
    Y = np.tile(jo.stoich_Y(om, 1.0).reshape((-1,) + (1,) * (len(shape) - 1)), (1,) + shape[1:])
    P[:, :6] = 30 * 101325.0
    T[:, :6] = 3000.0
    U, aux = jo.state_from_PTY(om, P, T, Y)
    U[1] += U[0] * rng.uniform(-50.0, 50.0, shape[1:])
    return U, jo.update_aux(om, U, aux)


def field_err(a, b):
    return max(np.sum(np.abs(a[i] - b[i])) / np.sum(np.abs(b[i])) for i in range(a.shape[0])
               if np.sum(np.abs(b[i])) > 1e-30)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["rk2_1d", "rk2_2d", "lf_source", "hllc_source", "rk2_hllc_source"])
def test_composed_steps_vs_oracle(case):
    from janc_b200.janc.simulation.set_simulator import Simulator
    from janc_b200.mechanism import DEFAULT_MECHANISM
    om = jo.load_mechanism(DEFAULT_MECHANISM)
    hllc = {"solver_type": "godunov", "interface_reconstruction": "WENO5_JS", "riemann_solver": "HLLC",
            "viscosity": "off"}
    dim = "1D" if case == "rk2_1d" else "2D"
    scheme = "RK2" if case.startswith("rk2") else "TVD_RK3"
    flux = hllc if "hllc" in case else None
    source = gravity if "source" in case else None
    cfg = _cfg(dim, scheme, flux, source)
    sim = Simulator(cfg)
    o = jo.Solver(om, dim, cfg["grid_config"]["dx"], cfg["grid_config"].get("dy"), cfg["boundary_config"], 0.4,
                  flux_config=cfg["flux_config"], time_scheme=scheme, source=source)
    U, aux = _state(om, dim)
    Ur, ar, t = U, aux, 0.0
    tr = 0.0
    for _ in range(4):
        U, aux, t, dt = sim.advance_func(U, aux, t, None)
        Ur, ar, tr, dtr = o.advance_func(Ur, ar, tr)
        assert abs(dt - dtr) <= 1e-12 * dtr
    assert np.all(np.isfinite(U))
    assert field_err(U, Ur) < 1e-12 and field_err(aux, ar) < 1e-12
