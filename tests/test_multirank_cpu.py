"""The multi-GPU path of bench.py without GPUs: two gloo ranks on the CPU
exercise the aggregation of a weak-scaling run (each rank its own lattice, the
job's time the slowest rank's, throughput summed over ranks)."""
from __future__ import annotations

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench

    ms = 2.0 + rank  # rank 1 is slower
    got_ms, value = bench.aggregate(ms, 1000.0, world, dist, "cpu")
    seeds = [None] * world
    dist.all_gather_object(seeds, bench.rank_seed(rank))
    q.put((rank, got_ms, value, seeds))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_aggregation():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got_ms, value, seeds in res:
        assert got_ms == 3.0  # the slowest rank
        assert value == pytest.approx(world * 1000.0 / 3.0e-3)
        assert len(set(seeds)) == world  # independent lattices


def test_single_rank_aggregation_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.aggregate(4.0, 500.0, 1) == (4.0, 500.0 / 4.0e-3)
