"""``jax.lax`` stand-in: the few control-flow and select primitives JANC uses."""
import numpy as _np


def while_loop(cond_fun, body_fun, init_val):
    val = init_val
    while bool(cond_fun(val)):
        val = body_fun(val)
    return val


def select(pred, on_true, on_false):
    from .numpy import _wrap
    return _wrap(_np.where(pred, on_true, on_false))


def cond(pred, true_fun, false_fun, *operands):
    return true_fun(*operands) if bool(pred) else false_fun(*operands)


def pmin(x, axis_name=None):
    return x


def axis_index(name):
    return 0


def ppermute(x, axis_name, perm):
    return x
