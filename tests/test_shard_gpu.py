"""Replica sharding of one ensemble (asd_ctx_set_ensemble / asd_ctx_shard_*):
two contexts on one GPU each hold part of the replicas, as two ranks would,
and their exchange is done here by adding the tensors (what the all-reduce
does).  The sharded S(q,t) must equal the unsharded context's: to 1e-12 in the
FP64 modes (only the connected-part term is formed differently: exactly
factorised in FP64 instead of per element), and within the split-precision
tolerance of the FP64 value in the split modes.  The stepped spins of each
shard equal the oracle's."""
from __future__ import annotations

import numpy as np
import pytest

import asd_b200 as asd
import oracle as orc
from asd_b200.shard import ShardedSqt, shard_range

pytestmark = pytest.mark.gpu

KW = dict(J1=-1.0, J2=0.2, alpha=0.05, h=(0.0, 0.0, 0.5), dt=0.005)


@pytest.mark.parametrize("N,nf,parts", [(16, 70, 2), (24, 33, 3), (12, 9, 2)])
def test_shards_add_up_to_the_whole_ensemble(oracle, N, nf, parts):
    import torch

    s0 = asd.random_spins(N, nf, seed=N + nf)
    M = N * N
    whole = asd.Context(asd.Params.make(N, nf, vx=2, vy=1, **KW))
    whole.set_spins(s0, as_origin=True)
    shards = []
    for r in range(parts):
        b, e = shard_range(nf, r, parts)
        c = asd.Context(asd.Params.make(N, e - b, vx=2, vy=1, **KW))
        c.set_spins(s0[b:e], as_origin=True)
        c.set_ensemble(nf)
        shards.append((b, e, c))
    f64 = dict(dtype=torch.float64, device="cuda")
    zs = [torch.zeros(3 * M, **f64) for _ in shards]
    for (_, _, c), z in zip(shards, zs):
        c.shard_origin_sums(z)
    ztot = sum(zs)
    for _, _, c in shards:
        c.shard_set_origin_sums(ztot)
    want_spins = s0
    for step in range(3):
        whole.step(1)
        want_spins = oracle.steps(orc.make_params(N, nf, **KW), want_spins, 1)
        for b, e, c in shards:
            c.step(1)
            assert np.array_equal(c.get_spins(), want_spins[b:e]), (step, b)
        ref = whole.sqt("fp64")
        for mode in ("fp64", "tf32x3", "bf16x3"):
            parts_t = [torch.zeros(2, **f64) for _ in shards]
            sums_t = [torch.zeros(3 * M, **f64) for _ in shards]
            for (_, _, c), p, s in zip(shards, parts_t, sums_t):
                c.shard_sqt_async(mode, p, s)
            out = torch.zeros(2, **f64)
            shards[0][2].shard_sqt_finish(sum(parts_t), sum(sums_t), out)
            torch.cuda.synchronize()
            got = complex(float(out[0]), float(out[1]))
            if mode.startswith("fp64"):
                assert abs(got - whole.sqt(mode)) <= 1e-12 * abs(ref), (step, mode)
            else:
                assert abs(got - ref) <= 1e-5 * abs(ref), (step, mode, got, ref)
    for _, _, c in shards:
        c.close()
    whole.close()


def test_sharded_helper_on_one_rank_equals_the_context():
    """ShardedSqt without a process group (one rank holding the whole
    ensemble) is the context's own S(q,t)."""
    import torch

    N, nf = 20, 40
    s0 = asd.random_spins(N, nf, seed=5)
    with asd.Context(asd.Params.make(N, nf, vx=1, vy=3, **KW)) as c:
        c.set_stream(torch.cuda.current_stream().cuda_stream)
        c.set_spins(s0, as_origin=True)
        ens = ShardedSqt(c, nf, N * N)
        ens.exchange_origin()
        for _ in range(2):
            c.step(1)
            ref = c.sqt("fp64")
            assert abs(ens.sqt("fp64") - ref) <= 1e-12 * abs(ref)
            assert abs(ens.sqt("tf32x3") - ref) <= 1e-5 * abs(ref)


def test_shard_entry_points_check_their_state():
    import torch

    with asd.Context(asd.Params.make(8, 4, **KW)) as c:
        with pytest.raises(asd.AsdError):
            c.set_ensemble(3)  # fewer than this shard's replicas
        c.set_spins(asd.random_spins(8, 4, seed=1), as_origin=True)
        c.set_ensemble(8)
        d = torch.zeros(3 * 64, dtype=torch.float64, device="cuda")
        two = torch.zeros(2, dtype=torch.float64, device="cuda")
        with pytest.raises(asd.AsdError):
            c.shard_sqt_finish(two, d, two)  # origin sums not exchanged yet
        c.shard_origin_sums(d)
        c.shard_set_origin_sums(d)
        c.set_spins(asd.random_spins(8, 4, seed=2), as_origin=True)
        with pytest.raises(asd.AsdError):
            c.shard_sqt_finish(two, d, two)  # a new origin needs a new exchange
