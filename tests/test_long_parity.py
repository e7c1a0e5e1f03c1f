"""Long and mid-size GPU parity against runs of the reference itself
(tests/golden/make_golden.py), through the C ABI:

* config 0 physics (2000 cells, slab = first 2 %, slip wall left, zero
  gradient right) at CFL 0.1 for 1000 steps: relative L1 per field at steps
  1, 10, 100 and 1000 <= 1e-12 (``fp64_strict``), <= 1e-10 (``fp64``); the
  mixed build <= 1e-4 on rho, p and T with the detonation front (largest
  cell with p > 2 atm) within one cell;
* the 2D channel at config-1 spacing, 128 x 64 cells with the seeded slab
  blobs, 200 steps at CFL 0.05: the same bars per field (rho, p, T and every
  Y_k), front per y row within one cell;
* the channel strip at CFL 0.1, where the reference's own step goes
  non-finite: the float64 builds fail at the same step and flag it;
* jb_u_to_prim (all outputs) and the state builder Solver.state_from_PTY
  against the reference's U_to_prim and initial states: bitwise in
  ``fp64_strict``, <= 1e-14 in ``fp64``.

Each test prints its measured errors on lines starting with ``PARITY``.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from janc_b200 import mechanism as jm  # noqa: E402
from janc_b200.solver import Solver  # noqa: E402

BC1 = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"}
BC2 = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient",
       "bottom_boundary": "slip_wall", "top_boundary": "slip_wall"}
TOL = {"fp64_strict": 1e-12, "fp64": 1e-10}


def G(golden_dir, name):
    return np.load(os.path.join(golden_dir, name + ".npz"))


def cuda(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


def rel_l1(a, b):
    return float(np.sum(np.abs(a - b)) / max(np.sum(np.abs(b)), 1e-300))


def _pressure(U, aux, nY):
    """p = rho R T with R from the state's mass fractions (get_R, N2 closing)."""
    invM = 1.0 / np.asarray(jm.load().tables["species_M"])
    rho = U[0]
    Y = U[nY:] / rho
    YN2 = 1.0 - np.sum(Y, axis=0)
    R = np.tensordot(invM[:8], Y, axes=1) + invM[8] * YN2
    return rho * R * aux[1]


def per_field(U, Uref, aux, auxref, nY):
    """Relative L1 of rho, p, T and each Y_k (species with any mass)."""
    out = {"rho": rel_l1(U[0], Uref[0]), "T": rel_l1(aux[1], auxref[1]),
           "p": rel_l1(_pressure(U, aux, nY), _pressure(Uref, auxref, nY))}
    for k in range(8):
        if np.sum(np.abs(Uref[nY + k])) > 1e-30:
            out[f"Y{k}"] = rel_l1(U[nY + k] / U[0], Uref[nY + k] / Uref[0])
    return out


def field_err(U, Uref):
    """Max over the conserved fields of the relative L1 error; the momentum
    components are measured together (sum of |d(rho u)| + |d(rho v)| over the
    sum of |rho u| + |rho v|), since a transverse momentum that is nearly zero
    everywhere has no meaningful relative error of its own."""
    nmom = 2 if U.ndim == 3 else 1
    mom = rel_l1(U[1:1 + nmom], Uref[1:1 + nmom])
    errs = [mom] + [rel_l1(U[i], Uref[i]) for i in [0] + list(range(1 + nmom, U.shape[0]))
                    if np.sum(np.abs(Uref[i])) > 1e-30]
    return max(errs)


def front(U, aux, nY):
    p = _pressure(U, aux, nY)
    if p.ndim == 2:
        return np.array([np.max(np.where(p[:, j] > 2 * 101325.0)[0], initial=-1) for j in range(p.shape[1])])
    return np.max(np.where(p > 2 * 101325.0)[0], initial=-1)


def _advance_checkpoints(s, g, checkpoints, cfl):
    """Advance from the fixture's initial state, returning the host state at
    each checkpoint step (one jb_advance call per segment) and all dts."""
    U, aux = cuda(g["U0"]), cuda(g["aux0"])
    out, dts, done = {}, [], 0
    for n in checkpoints:
        U, aux, dt = s.advance(U, aux, n - done, cfl=cfl)
        dts.append(host(dt))
        done = n
        out[n] = (host(U), host(aux))
    return out, np.concatenate(dts)


@pytest.mark.parametrize("prec", ["fp64_strict", "fp64", "mixed"])
def test_config0_1000_steps_vs_reference(prec, golden_dir):
    g = G(golden_dir, "config0_cfl01_1000")
    nx = g["U0"].shape[1]
    s = Solver(1, nx, dx=float(g["dx"]), boundary_config=BC1, precision=prec)
    cps = (1, 10, 100, 1000)
    res, dts = _advance_checkpoints(s, g, cps, float(g["cfl"]))
    assert s.status() == 0
    for n in cps:
        U, aux = res[n]
        Ur, auxr = g[f"U_{n}"], g[f"aux_{n}"]
        errs = per_field(U, Ur, aux, auxr, 3)
        df = int(front(U, aux, 3)) - int(front(Ur, auxr, 3))
        print(f"PARITY config0 cfl0.1 {prec} step {n}: max field {field_err(U, Ur):.3e} "
              + " ".join(f"{k} {v:.2e}" for k, v in errs.items()) + f" front {df:+d}")
        if prec == "mixed":
            assert errs["rho"] <= 1e-4 and errs["p"] <= 1e-4 and errs["T"] <= 1e-4, (n, errs)
            assert abs(df) <= 1, (n, df)
        else:
            assert field_err(U, Ur) <= TOL[prec], (n, field_err(U, Ur))
            assert field_err(aux, auxr) <= TOL[prec], n
            assert df == 0
    if prec != "mixed":
        np.testing.assert_allclose(dts, g["dts"], rtol=TOL[prec])


@pytest.mark.parametrize("prec", ["fp64_strict", "fp64", "mixed"])
def test_channel128x64_200_steps_vs_reference(prec, golden_dir):
    g = G(golden_dir, "channel128x64_200")
    nx, ny = g["U0"].shape[1:]
    d = float(g["dx"])
    s = Solver(2, nx, ny, d, d, BC2, precision=prec)
    cps = (1, 20, 200)
    res, dts = _advance_checkpoints(s, g, cps, float(g["cfl"]))
    assert s.status() == 0
    for n in cps:
        U, aux = res[n]
        Ur, auxr = g[f"U_{n}"], g[f"aux_{n}"]
        errs = per_field(U, Ur, aux, auxr, 4)
        df = np.max(np.abs(front(U, aux, 4) - front(Ur, auxr, 4)))
        print(f"PARITY channel128x64 cfl0.05 {prec} step {n}: max field {field_err(U, Ur):.3e} "
              + " ".join(f"{k} {v:.2e}" for k, v in errs.items()) + f" front max|d| {df}")
        if prec == "mixed":
            assert errs["rho"] <= 1e-4 and errs["p"] <= 1e-4 and errs["T"] <= 1e-4, (n, errs)
            assert df <= 1, (n, df)
        else:
            assert field_err(U, Ur) <= TOL[prec], (n, field_err(U, Ur))
            assert field_err(aux, auxr) <= TOL[prec], n
            assert df == 0
    if prec != "mixed":
        np.testing.assert_allclose(dts, g["dts"], rtol=TOL[prec])


@pytest.mark.parametrize("prec", ["fp64_strict", "fp64"])
def test_channel_strip_cfl01_goes_nonfinite_like_reference(prec, golden_dir):
    g = G(golden_dir, "cfl2d_strip")
    nx, ny = g["U0"].shape[1:]
    d = float(g["dx"])
    s = Solver(2, nx, ny, d, d, BC2, precision=prec)
    res, _ = _advance_checkpoints(s, g, (1, 10), 0.1)
    for n in (1, 10):
        U, aux = res[n]
        assert field_err(U, g[f"cfl0.1_U_{n}"]) <= TOL[prec], n
        assert field_err(aux, g[f"cfl0.1_aux_{n}"]) <= TOL[prec], n
    assert s.status() == 0
    bad = int(g["cfl0.1_first_nonfinite_step"])
    # the state before the reference's failing step is finite (its wave
    # speeds may already be NaN: that step's CFL dt is what goes non-finite)
    U, aux, _ = s.advance(cuda(g["U0"]), cuda(g["aux0"]), bad - 1, cfl=0.1)
    assert np.all(np.isfinite(host(U)))
    s.status()
    U, aux, _ = s.advance(U, aux, 1, cfl=0.1)
    assert not np.all(np.isfinite(host(U)))
    assert s.status() & 4
    print(f"PARITY channel strip cfl0.1 {prec}: non-finite at step {bad}, as the reference")


@pytest.mark.parametrize("prec", ["fp64_strict", "fp64"])
def test_u_to_prim_vs_reference(prec, golden_dir):
    g = G(golden_dir, "prim_si")
    cases = (("p2d", "bc2d_si", 2, None, ("rho", "u", "v", "Y", "p", "a")),
             ("p1d", "bc1d_si", 1, None, ("rho", "u", "Y", "p", "a")),
             ("prdc", "step2d_rdc", 2, {"P0": 10 * 101325, "T0": 300, "R0": 369, "x0": 0.08},
              ("rho", "u", "v", "Y", "p", "a")))
    for tag, fix, dim, nd, names in cases:
        b = G(golden_dir, fix)
        U = b["U_3"] if tag == "prdc" else b["U"]
        aux = b["aux_3"] if tag == "prdc" else b["aux"]
        if dim == 2:
            s = Solver(2, U.shape[1], U.shape[2], 1e-4, 1e-4, BC2, nondim_config=nd, precision=prec)
        else:
            s = Solver(1, U.shape[1], dx=1e-4, boundary_config=BC1, precision=prec)
        out = [host(t) for t in s.u_to_prim(cuda(U), cuda(aux))]
        for n, v in zip(names, out):
            ref = g[f"{tag}_{n}"]
            assert v.shape == ref.shape, (tag, n)
            if prec == "fp64_strict":
                np.testing.assert_array_equal(v, ref, err_msg=f"{tag} {n}")
            else:
                np.testing.assert_allclose(v, ref, rtol=1e-14, atol=0, err_msg=f"{tag} {n}")


def _state_inputs(golden_dir, which):
    """(P, T, Y) from which the reference built a step fixture's U0 / aux0:
    the stated pressures, T as stored in aux0, the stoichiometric mixture
    (H2:O2:N2 = 2:1:3.76 by mole with the mechanism's weights)."""
    W = {"H2": 2.016, "O2": 31.998, "N2": 28.014}
    m = {"H2": 2.0 * W["H2"], "O2": 1.0 * W["O2"], "N2": 3.76 * W["N2"]}
    tot = sum(m.values())
    Y0 = np.zeros(8)
    Y0[0], Y0[1] = m["H2"] / tot, m["O2"] / tot
    g = G(golden_dir, which)
    if which == "config0_cfl05":
        n = g["U0"].shape[1]
        P = np.full((1, n), 101325.0)
        P[:, :40] = 30 * 101325.0
        Y = np.tile(Y0[:, None], (1, n))
    else:
        nx, ny = g["U0"].shape[1:]
        P = np.full((1, nx, ny), 101325.0)
        P[:, :3] = 30 * 101325.0
        Y = np.tile(Y0[:, None, None], (1, nx, ny))
    return g, P, np.ascontiguousarray(g["aux0"][1:2]), np.ascontiguousarray(Y)


@pytest.mark.parametrize("prec", ["fp64_strict", "fp64"])
@pytest.mark.parametrize("which", ["config0_cfl05", "step2d_si"])
def test_state_from_PTY_vs_reference(prec, which, golden_dir):
    g, P, T, Y = _state_inputs(golden_dir, which)
    if which == "config0_cfl05":
        s = Solver(1, P.shape[1], dx=1e-4, boundary_config=BC1, precision=prec)
    else:
        s = Solver(2, P.shape[1], P.shape[2], 1e-4, 1e-4, BC2, precision=prec)
    U, aux = s.state_from_PTY(cuda(P), cuda(T), cuda(Y))
    U, aux = host(U), host(aux)
    if prec == "fp64_strict":
        np.testing.assert_array_equal(U, g["U0"])
        np.testing.assert_array_equal(aux, g["aux0"])
    else:
        np.testing.assert_allclose(U, g["U0"], rtol=1e-14, atol=0)
        np.testing.assert_allclose(aux, g["aux0"], rtol=1e-14, atol=0)
