"""CPU-only checks: the product's mechanism tables equal the reference's
golden tables, the C-ABI library loads and exports every function the header
declares, and host-side argument validation raises like the reference."""
import ctypes
import os
import re

import numpy as np
import pytest

import janc_b200
from janc_b200 import _native
from janc_b200 import mechanism as jm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "janc_b200.h")


@pytest.mark.parametrize("which,nd", [("si", None),
                                      ("rdc", {"P0": 10 * 101325, "T0": 300, "R0": 369, "x0": 0.08})])
def test_product_tables_equal_golden(which, nd, golden_dir):
    g = np.load(os.path.join(golden_dir, f"tables_{which}.npz"))
    m = jm.load(nondim_config=nd)
    for k in g.files:
        np.testing.assert_array_equal(np.squeeze(m.tables[k]), np.squeeze(g[k]), err_msg=k)


def test_pack_layout():
    p = jm.pack(jm.load())
    assert p.ns == 9 and p.nr == 8 and p.nreac == 19
    assert ctypes.sizeof(jm.MechParams) == janc_b200.lib().jb_sizeof_mech_params()
    assert p.pref == 101325.0 and p.T0 == 1.0


def _declared():
    src = open(HEADER).read()
    decl = r"^(?:int|long long|const char\*)\s+(jb_[A-Za-z0-9_]+)\s*\("
    return sorted(set(re.findall(decl, src, re.M)))


def test_library_exports_every_declared_symbol():
    L = janc_b200.lib()
    names = _declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_native.EXPORTS)


def test_version_and_null_handle_errors():
    L = janc_b200.lib()
    assert b"sm_100a" in L.jb_version()
    # argument checks happen before any device call
    assert L.jb_flux_func(None, None, None, 1.0, None, None) == 1
    assert L.jb_advance(None, None, None, None, None, 0.0, 0.0, 1, None, None) == 1
    assert L.jb_destroy(None) == 0
    bc = (ctypes.c_int * 4)(0, 0, 0, 0)
    h = ctypes.c_void_p()
    p = jm.pack(jm.load())
    assert L.jb_create(ctypes.byref(p), 3, 16, 16, 1.0, 1.0, bc, 0, ctypes.byref(h)) == 1   # bad dim
    assert L.jb_create(ctypes.byref(p), 2, 2, 16, 1.0, 1.0, bc, 0, ctypes.byref(h)) == 1    # too small
    bad = (ctypes.c_int * 4)(0, 9, 0, 0)
    assert L.jb_create(ctypes.byref(p), 2, 16, 16, 1.0, 1.0, bad, 0, ctypes.byref(h)) == 1  # bad bc
    assert L.jb_create(ctypes.byref(p), 2, 16, 16, 1.0, 1.0, bc, 7, ctypes.byref(h)) == 32  # precision


def test_config_errors_like_reference(tmp_path):
    with pytest.raises(AssertionError):
        jm.load(str(tmp_path / "mech.cti"))
    with pytest.raises(FileNotFoundError):
        jm.load(str(tmp_path / "missing.yaml"))


def test_stoichiometric_mixture():
    m = jm.load()
    Y = jm.stoichiometric_Y(m, 1.0)
    assert abs(Y[0] - 0.02852) < 1e-4 and abs(Y[1] - 0.22635) < 1e-4
