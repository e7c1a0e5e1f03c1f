"""The benchmark workloads at their full sizes on the GPU.

* Channel, 1024 x 256 (the bench's channel workload: 30 atm / 3000 K slab
  with 8 seeded +-5 % blobs, slip walls on all four sides, CFL 0.05): one
  step against the oracle (a NumPy restatement of
  src/janc_v2/simulation/set_simulator.py:410-447 that finishes one step of
  this grid in seconds) in every precision.
* Rotating-detonation annulus, 1600 x 1000 (the bench's rdc workload:
  periodic x, injector bottom, pressure outlet top, nondimensional): one
  step against the oracle in every precision (the oracle's step of this
  grid takes a minute or two).
* Size-independent properties of the same steps, over many steps:
  - mirror symmetry of the channel in x and in y (slip walls on both ends of
    each axis; the mirrored state has its normal momentum negated): WENO5-JS
    right-biased reconstruction is the left-biased one with the stencil
    reversed (reconstruction/WENO5_JS.py), the LF split swaps H+ and H- up to
    sign under the mirror, and every global reduction (alpha, the CFL
    minimum, the temperature solve's stop) sees the same set of values.  The
    reference's arithmetic (and the oracle's) is symmetric bit for bit, and
    so is the fp64_strict build; the fp64 and mixed builds' fluxes of a
    mirrored state differ from the mirrored fluxes by a few units in the last
    place of their arithmetic (float64, float32), which stays at round-off
    over the steps (relative L1 1e-12 for fp64, 1e-6 for mixed);
  - shift invariance of the rotating-detonation workload at 1600 x 1000
    (periodic in x; the reference's periodic pad is node-periodic,
    boundary/boundary_padding.py, so the distinct columns 0 .. nx-2 form a
    ring and column nx-1 repeats column 0): shifting the ring by k columns
    shifts every later state by k columns, bit for bit, through the injector
    and outlet strips (per column) and the global reductions.

Tolerances of the one-step comparison (relative L1 of the density, the
momentum vector, the energy, each species mass fraction and T):
fp64_strict 1e-12 (chemistry's 8 x 8 solve is LU-ordered differently from
LAPACK's), fp64 1e-10, mixed 1e-4 and 1e-6 on the density.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import bench  # noqa: E402  (the workload definitions)
from janc_b200.solver import Solver  # noqa: E402
from oracle import janc_oracle as jo  # noqa: E402

PRECS = ["fp64_strict", "fp64", "mixed"]
WALLS = {k: "slip_wall" for k in ("left_boundary", "right_boundary", "bottom_boundary", "top_boundary")}
BC_RDC = {"left_boundary": "periodic", "right_boundary": "periodic",
          "bottom_boundary": "rdc_injector", "top_boundary": "pressure_outlet"}
CFL_CH = bench.CFL_BY_WORKLOAD["channel"]
CFL_RDC = bench.CFL_BY_WORKLOAD["rdc"]


def _cuda(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def _l1(a, b):
    return float(np.sum(np.abs(a - b)) / np.sum(np.abs(b)))


def _errors(U, aux, Ur, auxr):
    """Relative L1 errors of the density, the momentum (as a vector: in the
    first step the y momentum of the slab is pure round-off of the balanced
    pressure faces, so only its size against the momentum matters), the
    energy, each species mass fraction with any mass, and T."""
    e = {"rho": _l1(U[0], Ur[0]), "mom": _l1(U[1:3], Ur[1:3]), "E": _l1(U[3], Ur[3]), "T": _l1(aux[1], auxr[1])}
    for k in range(8):
        if np.sum(np.abs(Ur[4 + k])) > 1e-30:
            e[f"Y{k}"] = _l1(U[4 + k] / U[0], Ur[4 + k] / Ur[0])
    return e


@pytest.fixture(scope="module")
def omech():
    from janc_b200.mechanism import DEFAULT_MECHANISM
    return jo.load_mechanism(DEFAULT_MECHANISM)


@pytest.fixture(scope="module")
def channel(omech):
    """Initial state of the channel workload and the oracle's first step."""
    P, T, Y = bench.c1_fields()
    U0, aux0 = jo.state_from_PTY(omech, P, T, Y)
    o = jo.Solver(omech, "2D", bench.LX / bench.NX, bench.LY / bench.NY, WALLS, CFL_CH)
    U1, aux1, _, dt = o.advance_func(U0, aux0, 0.0)
    return U0, aux0, U1, aux1, dt


def _channel_solver(prec):
    return Solver(2, bench.NX, bench.NY, bench.LX / bench.NX, bench.LY / bench.NY, WALLS, precision=prec)


@pytest.mark.parametrize("prec", PRECS)
def test_channel_full_size_step_vs_oracle(channel, prec):
    U0, aux0, U1, aux1, dt = channel
    s = _channel_solver(prec)
    Ug, ag, dts = s.advance(_cuda(U0), _cuda(aux0), 1, cfl=CFL_CH)
    torch.cuda.synchronize()
    assert s.status() == 0
    Ug, ag = Ug.cpu().numpy(), ag.cpu().numpy()
    tol = {"fp64_strict": 1e-12, "fp64": 1e-10, "mixed": 1e-4}[prec]
    assert abs(float(dts[0]) - dt) <= 1e-13 * dt
    err = _errors(Ug, ag, U1, aux1)
    assert max(err.values()) < tol, err
    assert err["rho"] < (1e-6 if prec == "mixed" else tol), err


@pytest.fixture(scope="module")
def rdc():
    """Initial state of the rotating-detonation workload, its theta and the
    oracle's first step."""
    from janc_b200.mechanism import DEFAULT_MECHANISM
    nm = jo.load_mechanism(DEFAULT_MECHANISM, bench.RDC_ND)
    P, T, Y, Yinj = bench.rdc_fields()
    theta = {"Yinj": Yinj, "Pb": 101325.0 / bench.RDC_ND["P0"]}
    U0, aux0 = jo.state_from_PTY(nm, P, T, Y)
    dx = 1e-4 / bench.RDC_ND["x0"]
    o = jo.Solver(nm, "2D", dx, dx, BC_RDC, CFL_RDC)
    U1, aux1, _, dt = o.advance_func(U0, aux0, 0.0, theta)
    return U0, aux0, theta, U1, aux1, dt


@pytest.mark.parametrize("prec", PRECS)
def test_rdc_full_size_step_vs_oracle(rdc, prec):
    U0, aux0, theta, U1, aux1, dt = rdc
    nx, ny = bench.RDC_NX, bench.RDC_NY
    dx = 1e-4 / bench.RDC_ND["x0"]
    s = Solver(2, nx, ny, dx, dx, BC_RDC, nondim_config=bench.RDC_ND, precision=prec)
    Ug, ag, dts = s.advance(_cuda(U0), _cuda(aux0), 1, cfl=CFL_RDC, theta=theta)
    torch.cuda.synchronize()
    assert s.status() == 0
    Ug, ag = Ug.cpu().numpy(), ag.cpu().numpy()
    tol = {"fp64_strict": 1e-12, "fp64": 1e-10, "mixed": 1e-4}[prec]
    assert abs(float(dts[0]) - dt) <= 1e-13 * dt
    err = _errors(Ug, ag, U1, aux1)
    assert max(err.values()) < tol, err
    assert err["rho"] < (1e-6 if prec == "mixed" else tol), err


def _mirror(U, aux, axis):
    """The state mirrored along x (axis 0) or y (axis 1), normal momentum negated."""
    Um = np.flip(U, axis=1 + axis).copy()
    Um[1 + axis] = -Um[1 + axis]
    return Um, np.flip(aux, axis=1 + axis).copy()


@pytest.mark.parametrize("prec", PRECS)
def test_channel_mirror_symmetry(prec, omech):
    P, T, Y = bench.c1_fields()
    U0, aux0 = jo.state_from_PTY(omech, P, T, Y)
    s = _channel_solver(prec)
    nsteps = 20
    U, aux, dts = s.advance(_cuda(U0), _cuda(aux0), nsteps, cfl=CFL_CH)
    U, aux, dts = U.cpu().numpy(), aux.cpu().numpy(), dts.cpu().numpy()
    assert np.isfinite(U).all() and s.status() == 0
    assert (U[0, :100] != U0[0, :100]).any()  # the slab has moved
    for axis in (0, 1):
        Um0, am0 = _mirror(U0, aux0, axis)
        Um, am, dtm = s.advance(_cuda(Um0), _cuda(am0), nsteps, cfl=CFL_CH)
        Um, am, dtm = Um.cpu().numpy(), am.cpu().numpy(), dtm.cpu().numpy()
        Ue, ae = _mirror(U, aux, axis)
        if prec == "fp64_strict":
            np.testing.assert_array_equal(dtm, dts)
            np.testing.assert_array_equal(Um, Ue)
            np.testing.assert_array_equal(am, ae)
        else:
            tol = 1e-12 if prec == "fp64" else 1e-6
            assert np.max(np.abs(dtm - dts) / dts) < tol
            err = _errors(Um, am, Ue, ae)
            assert max(err.values()) < tol, (axis, err)


def _ring_shift(a, k):
    """Shift the ring of distinct columns 0 .. nx-2 by k; column nx-1 repeats column 0."""
    r = np.roll(a[:, :-1], -k, axis=1)
    return np.concatenate([r, r[:, :1]], axis=1)


@pytest.mark.parametrize("prec", PRECS)
def test_rdc_full_size_shift_invariance(prec):
    P, T, Y, Yinj = bench.rdc_fields()
    for a in (P, T, Y):
        a[:, -1] = a[:, 0]  # node-periodic: the last column is the first one
    nx, ny = bench.RDC_NX, bench.RDC_NY
    dx = 1e-4 / bench.RDC_ND["x0"]
    s = Solver(2, nx, ny, dx, dx, BC_RDC, nondim_config=bench.RDC_ND, precision=prec)
    theta = {"Yinj": Yinj, "Pb": 101325.0 / bench.RDC_ND["P0"]}
    s.set_theta(theta)
    U0, aux0 = s.state_from_PTY(_cuda(P), _cuda(T), _cuda(Y))
    U0, aux0 = U0.cpu().numpy(), aux0.cpu().numpy()
    nsteps, k = 6, 357
    U, aux, dts = s.advance(_cuda(U0), _cuda(aux0), nsteps, cfl=CFL_RDC, theta=theta)
    U, aux, dts = U.cpu().numpy(), aux.cpu().numpy(), dts.cpu().numpy()
    assert np.isfinite(U).all() and s.status() == 0
    np.testing.assert_array_equal(U[:, -1], U[:, 0])
    Us, auxs, dtss = s.advance(_cuda(_ring_shift(U0, k)), _cuda(_ring_shift(aux0, k)), nsteps, cfl=CFL_RDC,
                               theta=theta)
    np.testing.assert_array_equal(dtss.cpu().numpy(), dts)
    np.testing.assert_array_equal(Us.cpu().numpy(), _ring_shift(U, k))
    np.testing.assert_array_equal(auxs.cpu().numpy(), _ring_shift(aux, k))
