"""parallel/boundary.py: the ghost-padded arrays of this rank's x slab
(neighbour columns through the ring, physical left / right conditions on the
first / last slab, bottom / top on every slab)."""
from ..boundary.boundary import boundary_conditions_1D, boundary_conditions_2D  # noqa: F401
