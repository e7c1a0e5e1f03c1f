"""Block-structured AMR step (src/janc_v2/simulation/time_step/TVD_RK3.py:15-36
with the vmapped block functions and the chemistry of
simulation/set_simulator.py:37-42, 97-113, 496-532).

The blocks' ghost layers come from a block layer (the external jaxamr
package in the reference, absent here); tests/golden/amr_blocks.py plays
that part for both the reference run that made tests/golden/amr_blocks.npz
(tests/golden/make_golden.py, group ``amr``) and the native path here.

* CPU: the oracle's AMR step equals the reference-run fixture bit for bit;
  configuration errors of the drop-in AMR wiring.
* GPU: the native AMR step (``AMR_Simulator`` of the drop-in mirror, one
  ``jb_amr_stage`` launch per stage and one ``jb_amr_chem``) against the
  fixture: <= 1e-12 relative L1 per field in every precision (the chemistry's
  8 x 8 solve is LU-ordered differently from LAPACK's, as in the single-grid
  step); its three SSP-RK3 stages alone (``TVD_RK3_amr``) against the
  oracle bitwise in fp64_strict; the block flux function and update_aux
  alone (``jb_amr_flux``, ``jb_amr_update_aux``) against the oracle bitwise
  in fp64_strict; the RK2 AMR form composed from them; argument checks.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

from oracle import janc_oracle as jo

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import amr_blocks  # noqa: E402

BC4 = {k: "slip_wall" for k in ("left_boundary", "right_boundary", "bottom_boundary", "top_boundary")}
LAYOUTS = (("b20", 2), ("b7x9", 1))


@pytest.fixture(scope="module")
def fx(golden_dir):
    return np.load(os.path.join(golden_dir, "amr_blocks.npz"))


@pytest.fixture(scope="module")
def mech(mech_path):
    return jo.load_mechanism(mech_path)


def _cfg(mech_path, precision, recon="WENO5_JS"):
    return {"thermo_config": {"thermo_model": "nasa7", "mechanism_directory": mech_path},
            "reaction_config": {"is_detailed_chemistry": True, "mechanism_directory": mech_path},
            "flux_config": {"solver_type": "flux_splitting", "interface_reconstruction": recon,
                            "split_method": "LF", "viscosity": "off"},
            "boundary_config": BC4, "time_config": {"temporal_evolution_scheme": "TVD_RK3", "dt": 1e-8},
            "precision": precision}


def _field_err(a, b):
    """Max over the nv + 2 fields of the relative L1 error (floor 1e-30)."""
    a, b = np.asarray(a), np.asarray(b)
    return max(float(np.sum(np.abs(a[:, f] - b[:, f])) / max(np.sum(np.abs(b[:, f])), 1e-30))
               for f in range(a.shape[1]))


# ---------------------------------------------------------------- CPU
@pytest.mark.parametrize("name,nsteps", LAYOUTS)
def test_oracle_amr_step_matches_reference(fx, mech, name, nsteps):
    nbx, nby, bx, by = (int(v) for v in fx[f"{name}_layout"])
    info = amr_blocks.info(nbx, nby)
    blk = fx[f"{name}_blk0"]
    for s in range(1, nsteps + 1):
        blk = jo.advance_one_step_amr(mech, amr_blocks, 1, blk, 1e-4, 1e-4, 1e-8, blk, info)
        assert np.array_equal(blk, fx[f"{name}_blk{s}"]), (name, s)


def test_amr_wiring_errors(mech_path):
    from janc_b200.janc.simulation import set_simulator as ss
    from janc_b200.janc.simulation import time_step as ts
    from janc_b200.janc import _state
    rc = {"is_detailed_chemistry": True, "mechanism_directory": mech_path}
    with pytest.raises(NotImplementedError):
        ss.set_rhs("1D", rc, None, False, True)
    old = dict(_state.config["flux"])
    try:
        _state.config["flux"] = {"solver_type": "godunov", "interface_reconstruction": "WENO5_JS",
                                 "riemann_solver": "HLLC", "viscosity": "off"}
        with pytest.raises(NotImplementedError):
            ss.set_rhs("2D", rc, None, False, True)
        _state.config["flux"] = old
        with pytest.raises(NotImplementedError):
            ss.set_rhs("2D", rc, {"self_defined_source_terms": lambda U, a, th: U}, False, True)
        ff, uf, sf = ss.set_rhs("2D", rc, None, False, True)
        with pytest.raises(KeyError):
            ss.set_advance_func("2D", old, rc, {"temporal_evolution_scheme": "Euler"}, True, ff, uf, sf)
        # no block layer: the jaxamr import fails before anything runs
        ts.set_amr_module(None)
        if "jaxamr" not in sys.modules:
            with pytest.raises(ImportError):
                ts.time_step_dict["TVD_RK3_amr"](1, None, 1.0, 1.0, 1e-8, None, None, None, ff, uf)
    finally:
        _state.config["flux"] = old


# ---------------------------------------------------------------- GPU
def _blocks_dev(a):
    import torch
    return torch.tensor(a, device="cuda", dtype=torch.float64)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64_strict", "fp64", "mixed"])
@pytest.mark.parametrize("name,nsteps", LAYOUTS)
def test_amr_simulator_matches_reference(fx, mech_path, precision, name, nsteps):
    import torch
    from janc_b200.janc.simulation import set_simulator as ss
    from janc_b200.janc.simulation import time_step as ts
    ts.set_amr_module(amr_blocks)
    try:
        adv_amr, _ = ss.AMR_Simulator(_cfg(mech_path, precision))
        nbx, nby, bx, by = (int(v) for v in fx[f"{name}_layout"])
        info = amr_blocks.info(nbx, nby)
        blk = _blocks_dev(fx[f"{name}_blk0"])
        for s in range(1, nsteps + 1):
            blk = adv_amr(1, blk, 1e-4, 1e-4, 1e-8, blk, info)
            ref = fx[f"{name}_blk{s}"]
            got = blk.cpu().numpy()
            assert _field_err(got, ref) < 1e-12, (name, s, _field_err(got, ref))
        torch.cuda.synchronize()
    finally:
        ts.set_amr_module(None)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["b20", "b7x9"])
def test_amr_rk3_stages_strict_bitwise(fx, mech, mech_path, name):
    """TVD_RK3_amr with the native block functions (one jb_amr_stage per
    stage) equals the oracle's restatement bit for bit in fp64_strict."""
    from janc_b200.janc.simulation import set_simulator as ss
    from janc_b200.janc.simulation import time_step as ts
    ss.AMR_Simulator(_cfg(mech_path, "fp64_strict"))
    ff, uf, _ = ss.set_rhs("2D", {"is_detailed_chemistry": True}, None, False, True)
    nbx, nby, bx, by = (int(v) for v in fx[f"{name}_layout"])
    info = amr_blocks.info(nbx, nby)
    blk0 = fx[f"{name}_blk0"]
    ts.set_amr_module(amr_blocks)
    try:
        b = _blocks_dev(blk0)
        got = ts.time_step_dict["TVD_RK3_amr"](1, b, 1e-4, 1e-4, 1e-8, b, info, None, ff, uf).cpu().numpy()
    finally:
        ts.set_amr_module(None)
    ref = jo.tvd_rk3_amr(mech, amr_blocks, 1, blk0, 1e-4, 1e-4, 1e-8, blk0, info)
    assert np.array_equal(got, ref), np.abs(got - ref).max()


@pytest.mark.gpu
def test_amr_block_functions_strict(fx, mech, mech_path):
    """jb_amr_flux and jb_amr_update_aux alone against the oracle's block
    functions (bitwise), on the ghost-padded blocks of the fixture's state."""
    import torch
    from janc_b200.solver import Solver
    nbx, nby, bx, by = (int(v) for v in fx["b20_layout"])
    info = amr_blocks.info(nbx, nby)
    G = amr_blocks.get_ghost_block_data(fx["b20_blk0"], info)
    U, aux = np.ascontiguousarray(G[:, :-2]), np.ascontiguousarray(G[:, -2:])
    s = Solver(2, 8, 8, 1.0, 1.0, {k: "periodic" for k in BC4}, jo_mech_to_native(mech_path),
               precision="fp64_strict")
    rhs = s.amr_flux(_blocks_dev(U), _blocks_dev(aux), 1e-4, 1e-4, 1e-8).cpu().numpy()
    assert np.array_equal(rhs, jo.amr_flux_func(mech, U, aux, 1e-4, 1e-4, 1e-8))
    U1 = U + rhs
    a1 = s.amr_update_aux(_blocks_dev(U1), _blocks_dev(aux)).cpu().numpy()
    assert np.array_equal(a1, jo.amr_update_func(mech, U1, aux))
    assert s.status() == 0
    torch.cuda.synchronize()


def jo_mech_to_native(mech_path):
    from janc_b200 import mechanism as jm
    return jm.load(mech_path)


@pytest.mark.gpu
def test_amr_rk2_composed(fx, mech, mech_path):
    """RK2.advance_one_step_amr composed from the native block functions
    against the same composition of the oracle's (RK2.py:14-32)."""
    from janc_b200.janc.simulation import set_simulator as ss
    from janc_b200.janc.simulation import time_step as ts
    cfg = _cfg(mech_path, "fp64_strict")
    cfg["time_config"]["temporal_evolution_scheme"] = "RK2"
    ts.set_amr_module(amr_blocks)
    try:
        adv_amr, _ = ss.AMR_Simulator(cfg)
        nbx, nby, bx, by = (int(v) for v in fx["b20_layout"])
        info = amr_blocks.info(nbx, nby)
        blk0 = fx["b20_blk0"]
        got = adv_amr(1, _blocks_dev(blk0), 1e-4, 1e-4, 1e-8, _blocks_dev(blk0), info).cpu().numpy()
    finally:
        ts.set_amr_module(None)
    g = amr_blocks.get_ghost_block_data(blk0, info)
    U, aux = g[:, :-2], g[:, -2:]
    dev = jo.amr_flux_func(mech, U, aux, 1e-4, 1e-4, 1e-8)
    U1 = U + dev
    a1 = jo.amr_update_func(mech, U1, aux)
    g1 = amr_blocks.get_ghost_block_data(np.concatenate([U1, a1], axis=1)[..., 3:-3, 3:-3], info)
    U1, a1 = g1[:, :-2], g1[:, -2:]
    dev1 = jo.amr_flux_func(mech, np.ascontiguousarray(U1), np.ascontiguousarray(a1), 1e-4, 1e-4, 1e-8)
    U2 = U + 1 / 2 * (dev + dev1)
    a2 = jo.amr_update_func(mech, U2, a1)
    b2 = np.concatenate([U2, a2], axis=1)[..., 3:-3, 3:-3]
    Ub, ab = b2[:, :-2], b2[:, -2:]
    dU = np.stack([jo.reaction_source_terms(mech, np.ascontiguousarray(Ub[b]), ab[b], 1e-8)
                   for b in range(Ub.shape[0])])
    Ub = Ub + dU
    ab = jo.amr_update_func(mech, Ub, ab)
    ref = np.concatenate([Ub, ab], axis=1)
    assert _field_err(got, ref) < 1e-13, _field_err(got, ref)


@pytest.mark.gpu
def test_amr_argument_checks(mech_path):
    import torch
    from janc_b200 import _native
    from janc_b200.solver import Solver
    lib = _native.lib()
    mechp = jo_mech_to_native(mech_path)
    s = Solver(2, 8, 8, 1.0, 1.0, {k: "periodic" for k in BC4}, mechp, precision="fp64")
    G = torch.zeros(2, 14, 26, 26, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(G.data_ptr())
    # out overlapping G, a bad stage, stage 2 without U0
    assert lib.jb_amr_stage(s._h, 2, 20, 20, 1e-4, 1e-4, 1, p, None, 1e-8, p, None) == 1
    assert lib.jb_amr_stage(s._h, 2, 20, 20, 1e-4, 1e-4, 4, p, None, 1e-8, None, None) == 1
    out = torch.empty_like(G)
    assert lib.jb_amr_stage(s._h, 2, 20, 20, 1e-4, 1e-4, 2, p, None, 1e-8, ctypes.c_void_p(out.data_ptr()),
                            None) == 1
    assert lib.jb_amr_chem(s._h, 1, 20, 20, p, -1.0, p, None) == 1
    # Godunov configuration: refused
    h = Solver(2, 8, 8, 1.0, 1.0, {k: "periodic" for k in BC4}, mechp, precision="fp64",
               flux_config={"solver_type": "godunov", "interface_reconstruction": "WENO5_JS",
                            "riemann_solver": "HLLC", "viscosity": "off"})
    assert lib.jb_amr_stage(h._h, 2, 20, 20, 1e-4, 1e-4, 1, p, None, 1e-8, ctypes.c_void_p(out.data_ptr()),
                            None) == 32
    # a 1D handle
    h1 = Solver(1, 8, None, 1.0, None, {"left_boundary": "periodic", "right_boundary": "periodic"}, mechp)
    assert lib.jb_amr_update_aux(h1._h, 1, 8, 8, p, p, ctypes.c_void_p(out.data_ptr()), None) == 1


@pytest.mark.gpu
def test_amr_muscl_stages_strict_bitwise(fx, mech, mech_path):
    """The block stages with MUSCL reconstruction (the handle's
    interface_reconstruction) against the oracle's block functions with
    MUSCL (whose MUSCL is pinned to the reference elsewhere), fp64_strict."""
    from janc_b200.janc.simulation import set_simulator as ss
    from janc_b200.janc.simulation import time_step as ts
    ss.AMR_Simulator(_cfg(mech_path, "fp64_strict", recon="MUSCL"))
    ff, uf, _ = ss.set_rhs("2D", {"is_detailed_chemistry": True}, None, False, True)
    nbx, nby, bx, by = (int(v) for v in fx["b20_layout"])
    info = amr_blocks.info(nbx, nby)
    blk0 = fx["b20_blk0"]
    ts.set_amr_module(amr_blocks)
    try:
        b = _blocks_dev(blk0)
        got = ts.time_step_dict["TVD_RK3_amr"](1, b, 1e-4, 1e-4, 1e-8, b, info, None, ff, uf).cpu().numpy()
    finally:
        ts.set_amr_module(None)
    ref = jo.tvd_rk3_amr(mech, amr_blocks, 1, blk0, 1e-4, 1e-4, 1e-8, blk0, info, recon="MUSCL")
    assert np.array_equal(got, ref), np.abs(got - ref).max()
