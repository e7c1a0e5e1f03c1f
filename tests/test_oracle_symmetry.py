"""Size-independent properties of the reference's step, checked on the
oracle (CPU): the GPU tests at the benchmarks' full sizes
(tests/test_full_size.py) rely on them.

* Mirror symmetry: a channel (and a 1D tube) with slip walls at both ends of each axis,
  mirrored in x or y with its normal momentum negated, steps to the mirror of
  the original's steps bit for bit (WENO5_JS.py's right-biased reconstruction
  is the left-biased one with the stencil reversed, and LF.py's split swaps
  H+ and H- up to sign under the mirror).
* Shift invariance: with node-periodic x (boundary_padding.py: the pad takes
  cells n-4 .. n-2 and 1 .. 3, so the distinct columns 0 .. n-2 form a ring
  and column n-1 repeats column 0), shifting the ring shifts every later
  state, through the rotating-detonation injector and outlet sides.
"""
import numpy as np
import pytest

import bench
from oracle import janc_oracle as jo

WALLS = {k: "slip_wall" for k in ("left_boundary", "right_boundary", "bottom_boundary", "top_boundary")}
BC_RDC = {"left_boundary": "periodic", "right_boundary": "periodic",
          "bottom_boundary": "rdc_injector", "top_boundary": "pressure_outlet"}


def _run(o, U, aux, n, theta=None):
    t = 0.0
    for _ in range(n):
        U, aux, t, _ = o.advance_func(U, aux, t, theta)
    return U, aux


def _mirror(U, axis, negate=True):
    Um = np.flip(U, 1 + axis).copy()
    if negate:
        Um[1 + axis] = -Um[1 + axis]
    return Um


@pytest.mark.parametrize("axis", [0, 1])
def test_oracle_channel_mirror_symmetry(axis):
    from janc_b200.mechanism import DEFAULT_MECHANISM
    om = jo.load_mechanism(DEFAULT_MECHANISM)
    P, T, Y = bench.c1_fields(nx=48, ny=24, slab=8)
    U0, a0 = jo.state_from_PTY(om, P, T, Y)
    rng = np.random.default_rng(5)
    U0[1] += U0[0] * 20.0 * rng.uniform(-1, 1, U0[0].shape)  # both signs of both velocities
    U0[2] += U0[0] * 20.0 * rng.uniform(-1, 1, U0[0].shape)
    a0 = jo.update_aux(om, U0, a0)
    o = jo.Solver(om, "2D", 1e-4, 1e-4, WALLS, 0.05)
    U, a = _run(o, U0, a0, 3)
    Um, am = _run(o, _mirror(U0, axis), _mirror(a0, axis, False), 3)
    np.testing.assert_array_equal(Um, _mirror(U, axis))
    np.testing.assert_array_equal(am, _mirror(a, axis, False))


def _ring_shift(a, k):
    r = np.roll(a[:, :-1], -k, axis=1)
    return np.concatenate([r, r[:, :1]], axis=1)


def test_oracle_rdc_ring_shift_invariance():
    from janc_b200.mechanism import DEFAULT_MECHANISM
    om = jo.load_mechanism(DEFAULT_MECHANISM, bench.RDC_ND)
    P, T, Y, Yinj = bench.rdc_fields(nx=64, ny=32)
    for a in (P, T, Y):
        a[:, -1] = a[:, 0]
    U0, a0 = jo.state_from_PTY(om, P, T, Y)
    dx = 1e-4 / bench.RDC_ND["x0"]
    o = jo.Solver(om, "2D", dx, dx, BC_RDC, 0.1)
    theta = {"Yinj": Yinj, "Pb": 101325.0 / bench.RDC_ND["P0"]}
    U, a = _run(o, U0, a0, 3, theta)
    np.testing.assert_array_equal(U[:, -1], U[:, 0])
    for k in (1, 17):
        Us, as_ = _run(o, _ring_shift(U0, k), _ring_shift(a0, k), 3, theta)
        np.testing.assert_array_equal(Us, _ring_shift(U, k))
        np.testing.assert_array_equal(as_, _ring_shift(a, k))


def test_oracle_tube_mirror_symmetry():
    """The 1D step (config-0 physics) of a tube with slip walls at both
    ends, mirrored with its velocity negated."""
    from janc_b200.mechanism import DEFAULT_MECHANISM
    om = jo.load_mechanism(DEFAULT_MECHANISM)
    n = 80
    rng = np.random.default_rng(8)
    P = np.full((1, n), 101325.0)
    T = 300.0 * (1 + 0.02 * rng.uniform(-1, 1, (1, n)))
    P[:, :6] = 30 * 101325.0
    T[:, :6] = 3000.0
    Y = np.tile(jo.stoich_Y(om, 1.0)[:, None], (1, n))
    U0, a0 = jo.state_from_PTY(om, P, T, Y)
    U0[1] += U0[0] * 20.0 * rng.uniform(-1, 1, U0[0].shape)
    a0 = jo.update_aux(om, U0, a0)
    o = jo.Solver(om, "1D", 5e-5, None, {"left_boundary": "slip_wall", "right_boundary": "slip_wall"}, 0.1)
    U, a = _run(o, U0, a0, 4)
    Um0 = U0[:, ::-1].copy()
    Um0[1] = -Um0[1]
    Um, am = _run(o, Um0, a0[:, ::-1].copy(), 4)
    Ue = U[:, ::-1].copy()
    Ue[1] = -Ue[1]
    np.testing.assert_array_equal(Um, Ue)
    np.testing.assert_array_equal(am, a[:, ::-1])
