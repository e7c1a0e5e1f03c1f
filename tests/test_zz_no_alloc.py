"""jb_update_aux_noalloc: the temperature solve for callers that cannot
allocate device memory (a plugin inside a host code that reserved all device
memory at start-up, or a call from inside another runtime's operator).  It
must give the same aux as jb_update_aux on a handle, call after call, while
its scratch comes from the library's static device array, and it must leave
the device's free memory unchanged.

The file name sorts last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from janc_b200 import _native  # noqa: E402
from janc_b200 import mechanism as jm  # noqa: E402
from janc_b200.solver import Solver  # noqa: E402

BC = {1: {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"},
      2: {k: "slip_wall" for k in ("left_boundary", "right_boundary", "bottom_boundary", "top_boundary")}}
GRID = {1: (5000, 1), 2: (96, 80)}  # within JB_NOALLOC_MAX_CELLS


def _state(s, dim, nx, ny, seed):
    """A burning-slab state with moving gas and a perturbed temperature guess."""
    rng = np.random.default_rng(seed)
    mech = jm.load()
    shape = (1, nx, ny) if dim == 2 else (1, nx)
    P = 101325.0 * (1 + 29 * (rng.uniform(size=shape) < 0.2))
    T = 300.0 + 2700.0 * rng.uniform(size=shape)
    Y0 = jm.stoichiometric_Y(mech, 1.0)
    Y = np.tile(Y0.reshape((-1,) + (1,) * dim), shape) * rng.uniform(0.6, 1.0, shape)
    vel = [rng.uniform(-500, 500, size=shape) for _ in range(dim)]
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")  # noqa: E731
    U, aux = s.state_from_PTY(t(P), t(T), t(Y), [t(v) for v in vel])
    guess = aux.clone()
    guess[1] *= torch.tensor(rng.uniform(0.9, 1.1, size=shape[1:]), device="cuda")
    return U, guess


def _call(L, params, dim, nx, ny, precision, U, guess, out, stream):
    return L.jb_update_aux_noalloc(ctypes.byref(params), dim, nx, ny, _native.PRECISION[precision],
                                   ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(guess.data_ptr()),
                                   ctypes.c_void_p(out.data_ptr()), stream)


@pytest.mark.parametrize("dim", [1, 2])
@pytest.mark.parametrize("precision", ["fp64", "fp64_strict"])
def test_noalloc_update_aux_matches_handle(precision, dim):
    nx, ny = GRID[dim]
    s = Solver(dim, nx, ny if dim == 2 else None, 1e-4, 1e-4 if dim == 2 else None, BC[dim], precision=precision)
    L = _native.lib()
    params = jm.pack(jm.load())
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call, seed in enumerate((11, 12)):  # two calls in a row share the static scratch
        U, guess = _state(s, dim, nx, ny, seed)
        ref = s.update_aux(U, guess)
        out = torch.full_like(guess, float("nan"))
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc = _call(L, params, dim, nx, ny, precision, U, guess, out, stream)
        assert rc == 0, (call, rc)
        torch.cuda.synchronize()
        if call > 0:  # the first call may load the library's device module
            assert torch.cuda.mem_get_info()[0] == free0, "the call changed the device's free memory"
        a, b = out.cpu().numpy(), ref.cpu().numpy()
        assert np.all(np.isfinite(a)), call
        if precision == "fp64_strict":
            np.testing.assert_array_equal(a, b, err_msg=f"call {call}")
        else:
            np.testing.assert_allclose(a, b, rtol=1e-12, atol=0.0, err_msg=f"call {call}")


def test_noalloc_refuses_mixed_precision():
    nx, ny = GRID[2]
    L = _native.lib()
    params = jm.pack(jm.load())
    U = torch.zeros((12, nx, ny), dtype=torch.float64, device="cuda")
    aux = torch.zeros((2, nx, ny), dtype=torch.float64, device="cuda")
    rc = _call(L, params, 2, nx, ny, "mixed", U, aux, aux, None)
    assert rc == 32  # JB_ERR_UNSUPPORTED, before any launch


def test_noalloc_rejects_grids_beyond_its_scratch():
    L = _native.lib()
    params = jm.pack(jm.load())
    n = int(np.sqrt(65536)) + 1  # (n x n) > JB_NOALLOC_MAX_CELLS
    U = torch.zeros((12, n, n), dtype=torch.float64, device="cuda")
    aux = torch.zeros((2, n, n), dtype=torch.float64, device="cuda")
    rc = _call(L, params, 2, n, n, "fp64", U, aux, aux, None)
    assert rc == 1  # JB_ERR_ARG, before any launch
