"""The per-cell temperature solve of the mixed-precision variant, restated
on the oracle (CPU), against the reference's global stopping rule
(thermo_model.py:135-153: all cells iterate while max|res| > tol and i < 5).

The per-cell rule (the kernels' halley_cell): a cell iterates while its own
|res| > tol, then takes one more Halley step (the step the global loop gives
every cell except the slowest) and stops; none if its residual is exactly 0
or NaN.  Every cell but the ones that set the global iteration count then
lands on the same converged temperature to round-off, and those differ by
at most tol / c_v (~1e-11 K in SI units).
"""
import numpy as np
import pytest

from oracle import janc_oracle as jo


def _get_T_per_cell(m, e, Y, T0):
    T = T0.copy()
    res, d1, d2, _ = jo._e_eqn(m, T, e, Y)
    active = np.ones(T.shape, bool)
    polished = np.zeros(T.shape, bool)
    for _ in range(jo.MAX_ITER):
        fresh = (np.abs(res) <= jo.TOL) & ~polished & (res != 0) & ~np.isnan(res)
        go = active & ((np.abs(res) > jo.TOL) | fresh)
        polished |= fresh & active
        if not go.any():
            break
        dT = -2 * res * d1 / (2 * (d1 * d1) - res * d2)
        T = np.where(go, T + dT, T)
        active = go
        res, d1, d2, _ = jo._e_eqn(m, T, e, Y)
    return T


@pytest.mark.parametrize("spread", [0.02, 0.3])
def test_per_cell_solve_matches_global_stop(spread):
    from janc_b200.mechanism import DEFAULT_MECHANISM
    m = jo.load_mechanism(DEFAULT_MECHANISM)
    rng = np.random.default_rng(23)
    n = 4000
    T_true = rng.uniform(300.0, 3500.0, (1, n))
    Y = np.tile(jo.stoich_Y(m, 1.0)[:8, None], (1, n)) * rng.uniform(0.5, 1.0, (8, n))
    Y[2:8] *= rng.uniform(0.0, 0.2, (6, n))  # some radicals and products
    e = jo._e_eqn(m, T_true, np.zeros_like(T_true), Y)[0]
    T0 = T_true * (1 + spread * rng.uniform(-1, 1, T_true.shape))
    T_glob = jo.get_T(m, e, Y, T0)[1:2]
    T_cell = _get_T_per_cell(m, e, Y, T0)
    cp, _, _, R, _ = jo.get_thermo(m, T_glob, Y)
    bound = jo.TOL / (cp - R) + 1e-14 * T_glob
    assert np.all(np.abs(T_cell - T_glob) <= bound)
    # and both solve the energy equation
    assert np.max(np.abs(T_cell - T_true) / T_true) < 1e-12
