"""``jax.numpy`` stand-in: NumPy functions whose array results carry a
functional ``.at[idx].set/multiply/add`` like JAX arrays.  Test infrastructure
only."""
import numpy as _np

from . import linalg  # noqa: F401


class _AtIndexer:
    def __init__(self, arr, idx):
        self.arr, self.idx = arr, idx

    def set(self, v):
        out = _np.array(self.arr, copy=True)
        out[self.idx] = _np.asarray(v)
        return _wrap(out)

    def multiply(self, v):
        out = _np.array(self.arr, copy=True)
        out[self.idx] = out[self.idx] * _np.asarray(v)
        return _wrap(out)

    def add(self, v):
        out = _np.array(self.arr, copy=True)
        out[self.idx] = out[self.idx] + _np.asarray(v)
        return _wrap(out)


class _At:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, idx):
        return _AtIndexer(self.arr, idx)


class JArr(_np.ndarray):
    @property
    def at(self):
        return _At(self)

    def block_until_ready(self):
        return self


def _wrap(x):
    if isinstance(x, _np.ndarray) and not isinstance(x, JArr):
        return x.view(JArr)
    return x


def _wrapped(fn):
    def g(*a, **k):
        r = fn(*a, **k)
        if isinstance(r, tuple):
            return tuple(_wrap(x) for x in r)
        return _wrap(r)
    g.__name__ = getattr(fn, "__name__", "f")
    return g


def array(x, dtype=None):
    return _wrap(_np.array(x, dtype=dtype))


asarray = array


def power(x, y):
    # JAX lowers an integer Python exponent to repeated multiplication
    # (lax.integer_pow); only the square occurs on the paths exercised here.
    if isinstance(y, int) and not isinstance(y, bool) and y == 2:
        x = _np.asarray(x)
        return _wrap(x * x)
    return _wrap(_np.power(x, y))


def clip(x, min=None, max=None):
    return _wrap(_np.clip(x, min, max))


def polyval(p, x):
    # Horner from zero, the scan JAX uses (same as numpy.polyval).
    p = _np.asarray(p)
    x = _np.asarray(x)
    y = _np.zeros_like(x)
    for c in p:
        y = y * x + c
    return _wrap(y)


def __getattr__(name):
    fn = getattr(_np, name)
    if callable(fn):
        return _wrapped(fn)
    return fn
