"""The batched persistent launch: many lattices of uneven sizes and
parameters in one cooperative, graph-captured kernel, against the FP32
oracle (oracle_steps_f32), bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

import asd_b200 as asd
import oracle as orc

pytestmark = pytest.mark.gpu


def ensemble(sizes, seed):
    rng = np.random.default_rng(seed)
    lats, spins = [], []
    for k, N in enumerate(sizes):
        alpha = float(rng.uniform(0.01, 0.2))
        kw = dict(J1=1.0, alpha=alpha, dt=0.01)
        if k % 3 == 1:
            kw.update(J2=-0.3)
        if k % 4 == 2:
            kw.update(h=(0.0, 0.1, 0.4))
        lats.append((N, kw))
        spins.append(asd.noisy_ordered_spins(N, float(rng.uniform(0.0, 0.5)), seed + k)
                     .astype(np.float32))
    return lats, spins


def check_bit_exact(oracle, lats, spins, b, nsteps):
    for l, ((N, kw), s) in enumerate(zip(lats, spins)):
        want = oracle.steps_f32(orc.make_params(N, 1, **kw), s, nsteps)
        got = b.get_spins(l)
        assert np.array_equal(got, want), (l, N, np.abs(got - want).max())


@pytest.mark.parametrize("tile,ctas", [(128, 2), (32, 1), (256, 4)])
def test_batch_bit_exact(oracle, tile, ctas):
    lats, spins = ensemble([48, 64, 37, 96, 5, 128, 160, 20], seed=3)
    with asd.Batch([asd.Lattice.make(N, **kw) for N, kw in lats]) as b:
        b.configure(tile, ctas)
        for l, s in enumerate(spins):
            b.set_spins(l, s)
        b.run(7)
        b.run(13)  # a second step count: a second captured graph
        check_bit_exact(oracle, lats, spins, b, 20)


@pytest.mark.parametrize("cluster,threads,sizes", [
    (8, 512, [48, 64, 37, 96, 5, 128, 160, 20]),   # 160^2 over 8 CTAs; 10 empty clusters
    (4, 256, [48, 64, 37, 5, 20, 3, 33]),
    (2, 512, [64, 37, 5, 20, 3]),
    (1, 512, [37, 5, 20, 3, 48]),                   # one CTA per lattice, whole lattices
    (6, 640, [160, 128, 96, 64, 48, 48]),           # a cluster size that is not a power of 2
    (3, 384, [96, 5, 37, 64, 3]),
])
def test_batch_cluster_bit_exact(oracle, cluster, threads, sizes):
    """The cluster-resident kernel (lattices in shared memory, rows split over
    a cluster's CTAs, halo rows through distributed shared memory) equals the
    FP32 oracle bit for bit, like the global-memory kernel."""
    lats, spins = ensemble(sizes, seed=4)
    with asd.Batch([asd.Lattice.make(N, **kw) for N, kw in lats]) as b:
        b.configure_cluster(cluster, threads)
        for l, s in enumerate(spins):
            b.set_spins(l, s)
        b.run(7)
        b.run(13)
        check_bit_exact(oracle, lats, spins, b, 20)
        b.configure(128, 2)  # switching kernels keeps the state
        b.run(3)
        check_bit_exact(oracle, lats, spins, b, 23)


def test_batch_cluster_rejects_a_batch_that_does_not_fit():
    """A 160^2 lattice needs 25600 sites (1.2 MB of shared memory) in one
    cluster: more than one CTA holds, and its rows are wider than 128
    threads."""
    with asd.Batch([asd.Lattice.make(160, J1=1.0, dt=0.01)]) as b:
        for size, threads in ((1, 640), (8, 128)):
            with pytest.raises(asd.AsdError) as e:
                b.configure_cluster(size, threads)
            assert e.value.code == asd.ASD_ERR_UNSUPPORTED
        b.configure_cluster(8, 512)


def test_batch_ensemble_configuration(oracle):
    """48 lattices with sizes drawn from {48, 64, 96, 128, 160}^2, noise
    amplitudes in [0, 0.5], alpha in [0.01, 0.2]; autotuned; 2000 steps.  The
    first 100 steps are checked bit for bit, the full run for unit length."""
    rng = np.random.default_rng(5)
    sizes = [int(x) for x in rng.choice([48, 64, 96, 128, 160], size=48)]
    lats, spins = ensemble(sizes, seed=11)
    with asd.Batch([asd.Lattice.make(N, **kw) for N, kw in lats]) as b:
        for l, s in enumerate(spins):
            b.set_spins(l, s)
        tile, ctas, ms = b.autotune(10)
        # tile 0: the cluster-resident kernel with clusters of `ctas` CTAs
        assert (tile in (32, 64, 128, 256) or (tile == 0 and 1 <= ctas <= 8)) and ctas >= 1
        assert ms > 0
        b.run(100)
        check_bit_exact(oracle, lats[:12], spins[:12], b, 100)
        b.run(1900)
        for l in range(len(lats)):
            s = b.get_spins(l)
            assert np.all(np.isfinite(s))
            assert np.allclose(np.linalg.norm(s.astype(np.float64), axis=-1), 1.0, atol=1e-6)


def test_fp32_constant_division_is_correctly_rounded():
    """The batched kernels divide by 3 and 6 with Markstein's correction step;
    over all 2^32 float bit patterns it must equal the correctly rounded
    division bit for bit (NaN = NaN), so the kernels still match the FP32
    oracle, which divides."""
    import torch

    bad = torch.zeros(1, dtype=torch.int64, device="cuda")
    asd.check_const_division_f32(bad.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(bad.item()) == 0
