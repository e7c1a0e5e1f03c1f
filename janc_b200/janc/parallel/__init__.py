"""x-slab decomposition (src/janc_v2/parallel): one slab per rank of the
initialised torch.distributed group, one process per GPU."""
