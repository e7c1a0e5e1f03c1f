"""Batched ensemble of 1D instances (one persistent kernel per call).

Every instance must take exactly the steps a single-case Solver takes on it
alone in the same precision (the kernels share their cell and tile bodies,
and the per-instance reductions are order independent), so the comparisons
against the Solver are exact; against the oracle the FP64 tolerance applies.
"""
import numpy as np
import pytest

from janc_b200 import mechanism as jm
from janc_b200.ensemble import ATM, detonation_tubes

BC1 = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"}


# ------------------------------------------------------------------ CPU only
def test_detonation_tubes_workload():
    tubes = detonation_tubes(64, seed=4)
    assert len(tubes) == 64
    nx = np.array([t["nx"] for t in tubes])
    assert nx.min() >= 1000 and nx.max() <= 16000
    phi = np.array([t["phi"] for t in tubes])
    Ti = np.array([t["T_ign"] for t in tubes])
    assert phi.min() >= 0.6 and phi.max() <= 1.4
    assert Ti.min() >= 2500 and Ti.max() <= 3500
    again = detonation_tubes(64, seed=4)
    assert [t["nx"] for t in again] == list(nx)
    t = tubes[0]
    ns = int(round(0.02 * t["nx"]))
    assert np.all(t["P"][0, :ns] == 30 * ATM) and np.all(t["P"][0, ns:] == ATM)
    assert np.all(t["T"][0, :ns] == t["T_ign"]) and np.all(t["T"][0, ns:] == 300.0)
    mech = jm.load(jm.DEFAULT_MECHANISM)
    np.testing.assert_allclose(t["Y"][:, 0], jm.stoichiometric_Y(mech, t["phi"]), rtol=0, atol=0)


# --------------------------------------------------------------------- GPU
def _small_tubes():
    """Ragged instances: tile edges misaligned, one instance shorter than a
    tile, different spacings, compositions and ignition states."""
    rng = np.random.default_rng(11)
    out = []
    for nx in (37, 300, 1000, 255, 2500):
        phi = rng.uniform(0.6, 1.4)
        Ti = rng.uniform(2500, 3500)
        ns = max(2, int(round(0.02 * nx)))
        P = np.full((1, nx), ATM)
        T = np.full((1, nx), 300.0)
        P[:, :ns] = 30 * ATM
        T[:, :ns] = Ti
        mech = jm.load(jm.DEFAULT_MECHANISM)
        Y = np.tile(jm.stoichiometric_Y(mech, phi)[:, None], (1, nx))
        out.append({"nx": nx, "dx": 0.1 / max(nx, 2000), "P": P, "T": T, "Y": Y})
    return out


def _ensemble(tubes, precision, cfl=0.1):
    from janc_b200.ensemble import Ensemble
    ens = Ensemble([t["nx"] for t in tubes], [t["dx"] for t in tubes], cfl=cfl, precision=precision)
    states = []
    for i, t in enumerate(tubes):
        U, aux = ens.state_from_PTY(t["P"], t["T"], t["Y"])
        ens.set_state(i, U, aux)
        states.append((U, aux))
    return ens, states


def _max_rel(a, b):
    a = a.detach().cpu().numpy()
    b = b.detach().cpu().numpy()
    errs = []
    for i in range(a.shape[0]):
        den = np.sum(np.abs(b[i]))
        if den > 1e-30:
            errs.append(np.sum(np.abs(a[i] - b[i])) / den)
    return max(errs)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ensemble_matches_single_solver(precision):
    import torch
    from janc_b200.solver import Solver
    tubes = _small_tubes()
    ens, states = _ensemble(tubes, precision)
    nsteps = 30
    dts = ens.advance(nsteps, record_dt=True)
    comb, per = ens.status()
    assert comb == 0, per
    n_exact = 0
    for i, t in enumerate(tubes):
        s = Solver(1, t["nx"], dx=t["dx"], boundary_config=BC1, precision=precision)
        U, aux, hist = s.advance(states[i][0], states[i][1], nsteps, cfl=0.1)
        Ue, auxe = ens.get_state(i)
        torch.cuda.synchronize()
        assert torch.all(torch.isfinite(Ue))
        assert _max_rel(Ue, U) <= 1e-12, i
        assert _max_rel(auxe, aux) <= 1e-12, i
        np.testing.assert_allclose(dts[i].cpu().numpy(), hist.cpu().numpy(), rtol=1e-12)
        n_exact += int(torch.equal(Ue, U) and torch.equal(auxe, aux))
    # the same cell and tile bodies and order-independent reductions: exact
    assert n_exact == len(tubes), f"bitwise equal instances: {n_exact} of {len(tubes)}"


def test_ensemble_outlet_needs_back_pressure():
    """An instance with a pressure outlet needs Pb (theta['Pb'] of the
    reference's boundary function); checked before any device work."""
    from janc_b200.ensemble import Ensemble
    with pytest.raises(KeyError):
        Ensemble([40, 50], [1e-4, 1e-4], boundary=[("slip_wall", "pressure_outlet"), ("slip_wall", "zero_gradient")])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ensemble_outlets_match_single_solver(precision):
    """Instances with pressure outlets on either side (the outlet ghost strips
    are written by the CTA that wrote the boundary cell in the mixed
    ensemble, by the select pass in the fp64 one) against the single-case
    Solver with the same back pressure."""
    import torch
    from janc_b200.ensemble import Ensemble
    from janc_b200.solver import Solver
    tubes = _small_tubes()[:4]
    pairs = [("slip_wall", "pressure_outlet"), ("pressure_outlet", "zero_gradient"),
             ("pressure_outlet", "pressure_outlet"), ("slip_wall", "zero_gradient")]
    Pb = [0.5 * ATM, 0.8 * ATM, 0.6 * ATM, 0.0]
    ens = Ensemble([t["nx"] for t in tubes], [t["dx"] for t in tubes], boundary=pairs, cfl=0.1,
                   precision=precision, Pb=Pb)
    states = []
    for i, t in enumerate(tubes):
        U, aux = ens.state_from_PTY(t["P"], t["T"], t["Y"])
        ens.set_state(i, U, aux)
        states.append((U, aux))
    nsteps = 30
    dts = ens.advance(nsteps, record_dt=True)
    comb, per = ens.status()
    assert comb == 0, per
    for i, t in enumerate(tubes):
        bc = {"left_boundary": pairs[i][0], "right_boundary": pairs[i][1]}
        s = Solver(1, t["nx"], dx=t["dx"], boundary_config=bc, precision=precision)
        U, aux, hist = s.advance(states[i][0], states[i][1], nsteps, cfl=0.1, theta={"Pb": Pb[i]})
        Ue, auxe = ens.get_state(i)
        torch.cuda.synchronize()
        assert torch.all(torch.isfinite(Ue))
        assert _max_rel(Ue, U) <= 1e-12, i
        assert _max_rel(auxe, aux) <= 1e-12, i
        np.testing.assert_allclose(dts[i].cpu().numpy(), hist.cpu().numpy(), rtol=1e-12)
        if "pressure_outlet" in pairs[i]:
            # the outlet has acted: the edge cell's pressure moved towards Pb
            x = 0 if pairs[i][0] == "pressure_outlet" else -1
            assert not torch.equal(Ue[:, x], states[i][0][:, x]), i


@pytest.mark.gpu
def test_ensemble_launch_shapes_agree():
    """The result does not depend on the block size or CTAs per SM, and two
    launches of 10 steps equal one of 20 (graph replay and restart)."""
    import torch
    tubes = _small_tubes()
    ref, _ = _ensemble(tubes, "mixed")
    ref.configure(128, 3)
    ref.advance(20)
    ref_states = [ref.get_state(i) for i in range(len(tubes))]
    for block, bpsm in ((64, 2), (256, 1), (128, 1)):
        ens, _ = _ensemble(tubes, "mixed")
        ens.configure(block, bpsm)
        ens.advance(10)
        ens.advance(10)
        torch.cuda.synchronize()
        for i in range(len(tubes)):
            U, aux = ens.get_state(i)
            assert torch.equal(U, ref_states[i][0]), (block, bpsm, i)
            assert torch.equal(aux, ref_states[i][1]), (block, bpsm, i)
    # the direct (non-graph) launch gives the same result
    ens, _ = _ensemble(tubes, "mixed")
    ens.advance(20, graph=False)
    torch.cuda.synchronize()
    for i in range(len(tubes)):
        assert torch.equal(ens.get_state(i)[0], ref_states[i][0])
    assert ref.launch_shape()["graph"] in ("stream capture", "explicit nodes")


@pytest.mark.gpu
def test_ensemble_fp64_vs_oracle():
    from oracle import janc_oracle as jo
    omech = jo.load_mechanism(jm.DEFAULT_MECHANISM)
    tubes = _small_tubes()[:2]
    ens, states = _ensemble(tubes, "fp64")
    nsteps = 8
    ens.advance(nsteps)
    for i, t in enumerate(tubes):
        o = jo.Solver(omech, "1D", t["dx"], None, BC1, 0.1)
        U, aux = states[i][0].cpu().numpy(), states[i][1].cpu().numpy()
        tt = 0.0
        for _ in range(nsteps):
            U, aux, tt, _dt = o.advance_func(U, aux, tt)
        Ue, auxe = ens.get_state(i)
        import torch
        assert _max_rel(Ue, torch.as_tensor(U)) < 1e-10
        assert _max_rel(auxe, torch.as_tensor(aux)) < 1e-10


@pytest.mark.gpu
def test_ensemble_autotune_restores_state():
    import torch
    tubes = _small_tubes()
    ens, _ = _ensemble(tubes, "mixed")
    before = [ens.get_state(i) for i in range(len(tubes))]
    best = ens.autotune(trial_steps=3)
    assert best["block"] in (64, 128, 256) and best["blocks_per_sm"] >= 1 and best["ms"] > 0
    shape = ens.launch_shape()
    assert shape["block"] == best["block"] and shape["blocks_per_sm"] == best["blocks_per_sm"]
    torch.cuda.synchronize()
    for i in range(len(tubes)):
        assert torch.equal(ens.get_state(i)[0], before[i][0])
        assert torch.equal(ens.get_state(i)[1], before[i][1])


@pytest.mark.gpu
def test_ensemble_barrier_timeout_is_reported():
    """A CTA group that waits for a CTA that never runs gives up after the
    wait limit and reports JB_ERR_TIMEOUT; the context stays usable."""
    import ctypes

    import torch
    from janc_b200 import _native
    tubes = _small_tubes()
    ens, _ = _ensemble(tubes, "mixed")
    comb = ctypes.c_uint()
    rc = ens._lib.jb_ens_selftest_timeout(ens._h, 20.0, ctypes.byref(comb),
                                          ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    assert comb.value & 16
    # the status was consumed; a fresh ensemble on the same context runs normally
    ens2, _ = _ensemble(tubes, "mixed")
    ens2.advance(3)
    assert ens2.status()[0] == 0
    assert _native.status_text(16) == "device wait timed out"
