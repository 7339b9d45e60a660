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


# --------------------------------------------------------- replica sharding
class _NumpyShard:
    """Stand-in for a context holding one shard of an ensemble, restating the
    shard contract of include/asd_b200.h in numpy (test infrastructure):
    part = (1/(M nfile_total)) sum_(f,c) (sum_i u_i S_t) (sum_j w_j S_0) over
    this shard's replicas, sums = per-site sums, finish = part - (1/M) sum_c U_c W_c
    from the ensemble's means."""

    def __init__(self, N, vx, vy, spin_t, spin_0):
        import numpy as np

        self.N, self.M = N, N * N
        idx = np.arange(self.M)
        th = 2 * np.pi * vx / N * (idx // N) + 2 * np.pi * vy / N * (idx % N)
        self.u, self.w = np.exp(-1j * th), np.exp(1j * th)
        self.t, self.o = spin_t, spin_0  # [nf_local][M][3]
        self.nft = None
        self.zs = None

    def set_ensemble(self, nft):
        self.nft = nft

    def shard_origin_sums(self, t):
        t.copy_(__import__("torch").from_numpy(self.o.sum(axis=0).reshape(-1)))

    def shard_set_origin_sums(self, t):
        self.zs = t.numpy().reshape(self.M, 3).copy()

    def shard_sqt_async(self, mode, part, sums):
        import numpy as np
        import torch

        F = np.einsum("i,fic->fc", self.u, self.t)
        G = np.einsum("j,fjc->fc", self.w, self.o)
        p = (F * G).sum() / (self.M * self.nft)
        part.copy_(torch.tensor([p.real, p.imag], dtype=torch.float64))
        sums.copy_(torch.from_numpy(self.t.sum(axis=0).reshape(-1)))

    def shard_sqt_finish(self, part, sums, out):
        import torch

        m = sums.numpy().reshape(self.M, 3) / self.nft
        z = self.zs / self.nft
        O = (self.u @ m) @ (self.w @ z)
        p = complex(float(part[0]), float(part[1])) - O / self.M
        out.copy_(torch.tensor([p.real, p.imag], dtype=torch.float64))


def _shard_worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "asd-kernel-fusion_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import oracle as orc
    from asd_b200.shard import ShardedSqt, shard_range

    N, nf, vx, vy = 6, 11, 2, 1
    s0 = orc.random_spins(N, nf, seed=3)
    st = orc.random_spins(N, nf, seed=4)
    b, e = shard_range(nf, rank, world)
    ens = ShardedSqt(_NumpyShard(N, vx, vy, st[b:e], s0[b:e]), nf, N * N, device="cpu")
    ens.exchange_origin()
    got = ens.sqt("fp64")
    q.put((rank, (b, e), got))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replica_sharded_sqt_equals_the_whole_ensemble(oracle):
    """Two gloo ranks, each holding part of one 11-replica ensemble, exchange
    their partial values and site sums: every rank's S(q,t) equals the
    oracle's S(q,t) of the whole ensemble (the OpenBLAS program's connected
    correlation, gemm/llg_sqt_mkl.c:349-423)."""
    import oracle as orc

    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [(0, 6), (6, 11)]
    s0 = orc.random_spins(6, 11, seed=3)
    st = orc.random_spins(6, 11, seed=4)
    want = oracle.sqt_gemm(6, 11, 2, 1, st, s0)
    for _, _, got in res:
        assert abs(got - want) <= 1e-12 * max(1.0, abs(want)), (got, want)


def test_shard_ranges_cover_the_ensemble():
    sys.path.insert(0, str(ROOT / "asd-kernel-fusion_b200"))
    from asd_b200.shard import shard_range

    for nf in (1, 7, 500, 1000):
        for world in (1, 2, 3, 8):
            r = [shard_range(nf, k, world) for k in range(world)]
            assert r[0][0] == 0 and r[-1][1] == nf
            assert all(r[k][1] == r[k + 1][0] for k in range(world - 1))
            assert max(e - b for b, e in r) - min(e - b for b, e in r) <= 1
