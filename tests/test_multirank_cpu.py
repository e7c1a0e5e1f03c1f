"""The replicas-only multi-GPU path of bench.py, exercised with two gloo
ranks on CPU: every rank reports its own device time, the job takes the
maximum, and the job throughput counts every rank's cells."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, times, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(dist, times[rank], device="cpu")
        val = bench.job_value(world, 1000, 5, ms)
        out[rank] = (ms, val)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_max_over_ranks_and_job_value_gloo():
    world = 2
    times = [12.5, 20.0]
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), times, out), nprocs=world, join=True)
    for r in range(world):
        ms, val = out[r]
        assert ms == 20.0
        assert val == pytest.approx(world * 1000 * 5 / 0.020)


def test_single_process_passthrough():
    assert bench.max_over_ranks(None, 3.0) == 3.0
    assert bench.job_value(1, 262144, 20, 20.0) == pytest.approx(262144 * 20 / 0.02)
