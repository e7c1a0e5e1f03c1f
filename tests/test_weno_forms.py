"""The WENO5-JS weight forms the kernels use, restated in NumPy and checked
against the reference's form (reconstruction/WENO5_JS.py, as the oracle
restates it) on CPU.

* The fp64 kernels' single-division form: alpha_k = C_k / (eps + IS_k)^2
  scaled by the product of all three (eps + IS_j)^2, so w_k is C_k times the
  product of the other two squares over their sum.
* The mixed kernels' paired float32 form: the split fluxes enter doubled
  (H' = F +- alpha q), the smoothness indicators as t^2 + 13/3 s^2 with eps
  scaled by 16 (16 (IS_k + eps) of the halved values), the weights as the
  squared ratios of the smallest eps + IS to each, and the linear weights
  folded into the candidate values; the face value is halved.

Both are the reference's weights in real arithmetic, so in float64 they
agree with it to round-off; in float32 the ratio form stays finite for SI
flux magnitudes (~1e11) and within float32 round-off of the reference.
"""
import numpy as np
import pytest

from oracle import janc_oracle as jo


def _single_division(a, b, c, d, e):
    t1, s1 = a - 4 * b + 3 * c, a - 2 * b + c
    t2, s2 = b - d, b - 2 * c + d
    t3, s3 = 3 * c - 4 * d + e, c - 2 * d + e
    e1 = 1e-6 + 0.25 * t1 * t1 + 13 / 12 * s1 * s1
    e2 = 1e-6 + 0.25 * t2 * t2 + 13 / 12 * s2 * s2
    e3 = 1e-6 + 0.25 * t3 * t3 + 13 / 12 * s3 * s3
    q1 = a / 3 - 7 / 6 * b + 11 / 6 * c
    q2 = -b / 6 + 5 / 6 * c + d / 3
    q3 = c / 3 + 5 / 6 * d - e / 6
    a1, a2, a3 = 0.1 * (e2 * e2 * e3 * e3), 0.6 * (e1 * e1 * e3 * e3), 0.3 * (e1 * e1 * e2 * e2)
    return (a1 * q1 + a2 * q2 + a3 * q3) / (a1 + a2 + a3)


def _paired_ratio(a, b, c, d, e):
    """Doubled inputs in, doubled face value out."""
    dt = a.dtype.type
    t1, s1 = c * dt(3) + (b * dt(-4) + a), (b * dt(-2) + a) + c
    t2, s2 = d * dt(-1) + b, (c * dt(-2) + b) + d
    t3, s3 = c * dt(3) + (d * dt(-4) + e), (d * dt(-2) + c) + e
    k13, e16 = dt(13 / 3), dt(16e-6)
    e1 = t1 * t1 + (s1 * k13 * s1 + e16)
    e2 = t2 * t2 + (s2 * k13 * s2 + e16)
    e3 = t3 * t3 + (s3 * k13 * s3 + e16)
    mn = np.minimum(e1, np.minimum(e2, e3))
    w1, w2, w3 = (mn / e1) ** 2, (mn / e2) ** 2, (mn / e3) ** 2
    q1 = c * dt(11 / 60) + (b * dt(-7 / 60) + a * dt(1 / 30))
    q2 = d * dt(0.2) + (c * dt(0.5) + b * dt(-0.1))
    q3 = e * dt(-0.05) + (d * dt(0.25) + c * dt(0.1))
    num = w3 * q3 + (w2 * q2 + w1 * q1)
    den = w3 * dt(0.3) + (w2 * dt(0.6) + w1 * dt(0.1))
    return num / den


def _stencils(scale, n=20000, seed=0):
    rng = np.random.default_rng(seed)
    f = rng.standard_normal((5, n)) * scale
    smooth = np.linspace(0, 1, 5)[:, None] * rng.standard_normal(n) * scale + scale
    f[:, : n // 4] = smooth[:, : n // 4]  # smooth (linear) stencils
    jump = rng.integers(1, 5, n)
    for i in range(n // 4, n // 2):  # one discontinuity
        f[jump[i]:, i] += 1e3 * scale
    return f


@pytest.mark.parametrize("scale", [1e-3, 1.0, 1e5, 1e11])
def test_weight_forms_match_the_reference_in_float64(scale):
    f = _stencils(scale)
    ref_L = jo._weno_L(*f)
    ref_R = jo._weno_R(*f)
    top = np.max(np.abs(f), axis=0)
    np.testing.assert_array_less(np.abs(_single_division(*f) - ref_L), 1e-12 * top + 1e-300)
    np.testing.assert_array_less(np.abs(0.5 * _paired_ratio(*(2 * f)) - ref_L), 1e-12 * top + 1e-300)
    # the right-biased value is the left-biased one of the reversed stencil
    np.testing.assert_array_less(np.abs(0.5 * _paired_ratio(*(2 * f[::-1])) - ref_R), 1e-12 * top + 1e-300)


@pytest.mark.parametrize("scale", [1.0, 1e5, 1e11])
def test_paired_ratio_form_in_float32(scale):
    f = _stencils(scale, seed=1)
    with np.errstate(over="raise", invalid="raise"):
        got = 0.5 * _paired_ratio(*(2 * f).astype(np.float32))
    assert np.all(np.isfinite(got))
    top = np.max(np.abs(f), axis=0)
    err = np.abs(got.astype(np.float64) - jo._weno_L(*f))
    assert np.all(err <= 1e-5 * top)
