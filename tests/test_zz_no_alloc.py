"""jb_update_aux_noalloc: the temperature solve for callers that cannot
allocate device memory (a plugin inside a host code that reserved all device
memory at start-up, or a call from inside another runtime's operator).  It
must give the same aux as jb_update_aux on a handle, call after call, while
its scratch comes from the library's static device array.

The file name sorts last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from janc_b200 import _native  # noqa: E402
from janc_b200 import mechanism as jm  # noqa: E402
from janc_b200.solver import Solver  # noqa: E402


def _state(s, nx, ny, seed):
    """A burning-slab state with moving gas and a perturbed temperature guess."""
    rng = np.random.default_rng(seed)
    mech = jm.load()
    P = 101325.0 * (1 + 29 * (rng.uniform(size=(1, nx, ny)) < 0.2))
    T = 300.0 + 2700.0 * rng.uniform(size=(1, nx, ny))
    Y = np.tile(jm.stoichiometric_Y(mech, 1.0)[:, None, None], (1, nx, ny)) * rng.uniform(0.6, 1.0, (1, nx, ny))
    vel = [rng.uniform(-500, 500, size=(1, nx, ny)) for _ in range(2)]
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")  # noqa: E731
    U, aux = s.state_from_PTY(t(P), t(T), t(Y), [t(v) for v in vel])
    guess = aux.clone()
    guess[1] *= torch.tensor(rng.uniform(0.9, 1.1, size=(nx, ny)), device="cuda")
    return U, guess


@pytest.mark.parametrize("precision", ["fp64", "fp64_strict"])
def test_noalloc_update_aux_matches_handle(precision):
    nx, ny = 96, 80  # 7680 cells, within JB_NOALLOC_MAX_CELLS
    bc = {k: "slip_wall" for k in ("left_boundary", "right_boundary", "bottom_boundary", "top_boundary")}
    s = Solver(2, nx, ny, 1e-4, 1e-4, bc, precision=precision)
    L = _native.lib()
    params = jm.pack(jm.load())
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call, seed in enumerate((11, 12)):  # two calls in a row share the static scratch
        U, guess = _state(s, nx, ny, seed)
        ref = s.update_aux(U, guess)
        out = torch.full_like(guess, float("nan"))
        rc = L.jb_update_aux_noalloc(ctypes.byref(params), 2, nx, ny, _native.PRECISION[precision],
                                     ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(guess.data_ptr()),
                                     ctypes.c_void_p(out.data_ptr()), stream)
        assert rc == 0, (call, rc)
        torch.cuda.synchronize()
        a, b = out.cpu().numpy(), ref.cpu().numpy()
        assert np.all(np.isfinite(a)), call
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=0.0, err_msg=f"call {call}")


def test_noalloc_rejects_grids_beyond_its_scratch():
    L = _native.lib()
    params = jm.pack(jm.load())
    n = int(np.sqrt(65536)) + 1  # (n x n) > JB_NOALLOC_MAX_CELLS
    U = torch.zeros((12, n, n), dtype=torch.float64, device="cuda")
    aux = torch.zeros((2, n, n), dtype=torch.float64, device="cuda")
    rc = L.jb_update_aux_noalloc(ctypes.byref(params), 2, n, n, 1, ctypes.c_void_p(U.data_ptr()),
                                 ctypes.c_void_p(aux.data_ptr()), ctypes.c_void_p(aux.data_ptr()), None)
    assert rc == 1  # JB_ERR_ARG, before any launch
