"""x-slab decomposition of one grid over the ranks of a process group.

The reference's parallel mode (``computation_config['is_parallel']``,
src/janc_v2/parallel/) splits the x axis into equal slabs, one per device
(grid_partion.py ``split_and_distribute_grid``), and before every flux
evaluation exchanges 3 ghost columns of ``U || aux`` with both x neighbours
through a ring permutation (boundary_padding.py ``exchange_halo``); the first
and last slab then apply the physical left / right boundary conditions
(parallel/boundary.py), every slab its bottom / top ones; the CFL time step is
the minimum over the devices (``jax.lax.pmin`` in set_simulator.py:413-436).
The LF wave speed and the temperature solve's stopping test stay per slab.

Here each rank is one process with one GPU.  ``Slab`` names this rank's
place in the decomposition; ``SlabExchange`` is the transport behind the
native library's ``jb_set_exchange`` hook: the library packs its edge columns
and the CFL pair on the launch stream and calls back here between kernels;
the ring exchange and the MIN all-reduce go through ``torch.distributed``
(NCCL on device buffers, or gloo through host copies), stream-ordered on the
launch stream.  The halo buffer the callback fills is read directly by the
stencil kernels, so no padded copy of the slab is ever formed.
"""
import ctypes

import torch
import torch.distributed as dist

from . import _native

HALO_WIDTH = 3


class Slab:
    """This rank's slab: ``rank`` of ``size`` along x within ``group``.

    Defaults to the default process group's rank and size."""

    def __init__(self, group=None, rank=None, size=None):
        self.group = group
        if rank is None or size is None:
            if not (dist.is_available() and dist.is_initialized()):
                raise RuntimeError("Slab needs an initialised torch.distributed process group "
                                   "(or explicit rank and size)")
            rank = dist.get_rank(group) if rank is None else rank
            size = dist.get_world_size(group) if size is None else size
        if not 0 <= rank < size:
            raise ValueError(f"rank {rank} outside a group of {size}")
        self.rank, self.size = int(rank), int(size)

    @property
    def left(self):
        """Group rank of the left neighbour (ring order, as exchange_halo)."""
        return (self.rank - 1) % self.size

    @property
    def right(self):
        return (self.rank + 1) % self.size

    def global_rank(self, r):
        return dist.get_global_rank(self.group, r) if self.group is not None else r

    def boundary_kinds(self, kinds):
        """Native side kinds of this slab from the global domain's: an x side
        inside the domain, or any x side of a periodic x axis, is a halo
        side; the domain's own left / right conditions stay on the first /
        last slab (parallel/boundary.py:18-25).  Bottom / top are unchanged."""
        out = list(kinds)
        periodic = _native.BC_KIND["periodic"]
        if self.rank > 0 or kinds[0] == periodic:
            out[0] = _native.BC_HALO
        if self.rank < self.size - 1 or kinds[1] == periodic:
            out[1] = _native.BC_HALO
        return out

    def columns(self, nx_global):
        """(first column, count) of this slab; nx must divide evenly, as
        split_and_distribute_grid asserts."""
        if nx_global % self.size:
            raise AssertionError("nx should be divisible by number of avaliable devices")
        n = nx_global // self.size
        return self.rank * n, n


def split_and_distribute_grid(grid, slab, split_axis=1, device=None):
    """This rank's slab of a global array (grid_partion.py:7-12): the
    ``slab.rank``-th of ``slab.size`` equal chunks along ``split_axis``, as a
    contiguous tensor on ``device`` (the current CUDA device by default)."""
    t = torch.as_tensor(grid)
    if t.shape[split_axis] % slab.size:
        raise AssertionError("nx should be divisible by number of avaliable devices")
    chunk = torch.chunk(t, slab.size, dim=split_axis)[slab.rank]
    dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
    return chunk.to(device=dev, dtype=torch.float64).contiguous()


def gather_grid(local, slab, gather_axis=1):
    """The global array from every rank's slab (grid_partion.py:14-15),
    on every rank (an all-gather over the slab's group)."""
    parts = [torch.empty_like(local) for _ in range(slab.size)]
    backend = dist.get_backend(slab.group)
    if backend == "gloo" and local.is_cuda:
        host = [torch.empty_like(local, device="cpu") for _ in range(slab.size)]
        dist.all_gather(host, local.cpu(), group=slab.group)
        parts = [h.to(local.device) for h in host]
    else:
        dist.all_gather(parts, local.contiguous(), group=slab.group)
    return torch.cat(parts, dim=gather_axis)


class SlabExchange:
    """Halo and CFL transport of one native handle (``jb_set_exchange``).

    Buffers (device): ``send`` and ``halo`` [2][nv+2][3][ny] (side 0 the left
    x side, side 1 the right), ``red`` the int64 CFL pair.  The ring: this
    rank's ``send[1]`` (columns nx-3..nx-1) becomes the right neighbour's
    ``halo[0]``, ``send[0]`` (columns 0..2) the left neighbour's ``halo[1]``."""

    def __init__(self, slab, nv, ny, device):
        self.slab = slab
        shape = (2, nv + 2, HALO_WIDTH, ny)
        self.send = torch.zeros(shape, dtype=torch.float64, device=device)
        self.halo = torch.zeros(shape, dtype=torch.float64, device=device)
        self.red = torch.zeros(2, dtype=torch.int64, device=device)
        self.error = None
        self.calls = 0
        self._host = None
        if slab.size > 1 or slab.group is not None:
            self._host = dist.get_backend(slab.group) == "gloo"
        self._fn = _native.EXCHANGE_FN(self._callback)

    def attach(self, lib, handle):
        def p(t):
            return ctypes.c_void_p(t.data_ptr())
        _native.check(lib.jb_set_exchange(handle, p(self.send), p(self.halo), p(self.red), self._fn, None),
                      handle, "jb_set_exchange")

    # ------------------------------------------------------------ transport
    def _callback(self, user, flags, stream):
        """The jb_exchange_fn: 0 on success; any failure (a peer that left, a
        process-group timeout) is kept in ``error`` and returned as 1, which
        the library reports as a failed call (no GPU wait is involved: the
        transport blocks on the host)."""
        try:
            if self.send.is_cuda and stream and torch.cuda.current_stream(self.send.device).cuda_stream != stream:
                with torch.cuda.stream(torch.cuda.ExternalStream(stream, device=self.send.device)):
                    self.transfer(flags)
            else:
                self.transfer(flags)
            self.calls += 1
            return 0
        except BaseException as e:  # the C side reports a failed transport
            self.error = e
            return 1

    def transfer(self, flags):
        s = self.slab
        if flags & _native.XCH_DT and s.size > 1:
            if self._host:
                r = self.red.cpu()
                dist.all_reduce(r, op=dist.ReduceOp.MIN, group=s.group)
                self.red.copy_(r)
            else:
                dist.all_reduce(self.red, op=dist.ReduceOp.MIN, group=s.group)
        if flags & _native.XCH_HALO:
            if s.size == 1:  # the ring closes on itself (a periodic x axis on one device)
                self.halo[0].copy_(self.send[1])
                self.halo[1].copy_(self.send[0])
                return
            send, halo = (self.send.cpu(), torch.empty_like(self.halo, device="cpu")) if self._host \
                else (self.send, self.halo)
            ops = [dist.P2POp(dist.isend, send[1], s.global_rank(s.right), s.group, tag=0),
                   dist.P2POp(dist.irecv, halo[0], s.global_rank(s.left), s.group, tag=0),
                   dist.P2POp(dist.isend, send[0], s.global_rank(s.left), s.group, tag=1),
                   dist.P2POp(dist.irecv, halo[1], s.global_rank(s.right), s.group, tag=1)]
            for req in dist.batch_isend_irecv(ops):
                req.wait()
            if self._host:
                self.halo.copy_(halo)
