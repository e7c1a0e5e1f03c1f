"""grid_partion.py: split a global array into x slabs and gather it back.
The reference places every slab on its own device of one process
(jax.device_put_sharded); here each rank process keeps its own slab."""
from ...slab import Slab
from ...slab import gather_grid as _gather
from ...slab import split_and_distribute_grid as _split
from .. import _state


def _slab():
    s = _state.config["slab"]
    if s is None:
        s = _state.config["slab"] = Slab()
    return s


def split_and_distribute_grid(grid, split_axis=1):
    """This rank's equal chunk of ``grid`` along ``split_axis`` (an
    AssertionError when it does not divide evenly), on this rank's GPU."""
    return _split(grid, _slab(), split_axis)


def gather_grid(sharded_grid, gather_axis=1):
    """The global array from every rank's slab, on every rank."""
    return _gather(sharded_grid, _slab(), gather_axis)
