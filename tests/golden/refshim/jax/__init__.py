"""NumPy-backed stand-in for the small part of JAX that JANC's ``janc_v2``
package touches, so the reference's own Python source can be executed in a
container without JAX to produce golden vectors.

Test infrastructure only (used by ``tests/golden/make_golden.py``).  It is not
a JAX implementation: ``jit``/``pmap`` are identities, ``vmap`` is a Python
loop that stacks results, ``lax.while_loop`` is a Python ``while``, and
``custom_vjp`` only records the rules.  Arithmetic is IEEE-754 float64 through
NumPy, i.e. what ``jax_enable_x64`` gives on a CPU backend up to libm ulps.
"""
import numpy as _np

from . import numpy  # noqa: F401  (jax.numpy)
from . import lax  # noqa: F401
from .numpy import _wrap


class _Config:
    def update(self, *a, **k):
        pass


config = _Config()


def devices():
    return ["cpu:0"]


def jit(f=None, **kw):
    if f is None:
        return lambda g: g
    return f


def pmap(f, *a, **k):
    return f


def vmap(f, in_axes=0, out_axes=0):
    """Loop-and-stack vmap over the (single) mapped length."""
    def g(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = None
        for a, ax in zip(args, axes):
            if ax is not None:
                n = _np.shape(a)[ax]
                break
        outs = []
        for i in range(n):
            sl = [(_np.take(a, i, axis=ax) if ax is not None else a) for a, ax in zip(args, axes)]
            sl = [(_wrap(s) if isinstance(s, _np.ndarray) else s) for s in sl]
            outs.append(f(*sl))
        if isinstance(outs[0], tuple):
            return tuple(_wrap(_np.stack([_np.asarray(o[j]) for o in outs], axis=out_axes))
                         for j in range(len(outs[0])))
        return _wrap(_np.stack([_np.asarray(o) for o in outs], axis=out_axes))
    return g


class custom_vjp:
    def __init__(self, fun):
        self.fun = fun
        self.fwd = None
        self.bwd = None

    def __call__(self, *a, **k):
        return self.fun(*a, **k)

    def defvjp(self, fwd, bwd):
        self.fwd, self.bwd = fwd, bwd
