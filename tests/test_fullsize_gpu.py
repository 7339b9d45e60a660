"""The configurations at their full sizes: the 128 x 128 lattice with 500
replicas (J = -1, h = (0, 0, 0.5), alpha = 0.05, dt = 0.005; S(q,t) in TF32x3
and FP64) and the 256 x 256 lattice with 1000 replicas (J = 1, J2 = -0.3,
alpha = 0.02, dt = 0.005; S(q,t) in BF16x3 and FP64).

* One RK4 step against the oracle, bit for bit, through every way of
  stepping: the one-launch kernel, the stage kernels, the default choice, and
  the host-buffer steps (synchronous and pipelined).
* Properties that hold at any size: the step commutes with a translation of
  the periodic lattice and with a permutation of the replicas, bit for bit,
  and the renormalised spins have the set length.
* S(q,t): the FP64 GEMM path against the oracle's factorised form (1e-12),
  the split modes within 1e-5 of the FP64 path.
* Known answers at 256 x 256 x 1000: a uniform ferromagnet is stationary and
  identical replicas have no connected correlation.
* A lattice whose GEMM has more than 2^31 tiles (N = 2900).
"""
from __future__ import annotations

import numpy as np
import pytest

import asd_b200 as asd
import oracle as orc

pytestmark = pytest.mark.gpu

CONFIGS = {
    "128x128x500": (128, 500, dict(J1=-1.0, alpha=0.05, h=(0.0, 0.0, 0.5), dt=0.005),
                    ["fp64", "tf32x3", "bf16x3", "fp16x3"]),
    "256x256x1000": (256, 1000, dict(J1=1.0, J2=-0.3, alpha=0.02, dt=0.005),
                     ["fp64", "bf16x3", "tf32x3", "fp16x3"]),
}


def roll(s, N, dr, dc):
    """Periodic translation of every replica's lattice by (dr, dc)."""
    nf = s.shape[0]
    return np.ascontiguousarray(np.roll(s.reshape(nf, N, N, 3), (dr, dc), axis=(1, 2))
                                .reshape(nf, N * N, 3))


@pytest.fixture(scope="module", params=list(CONFIGS))
def case(request, oracle):
    N, nf, kw, modes = CONFIGS[request.param]
    s0 = asd.random_spins(N, nf, seed=3)
    want = oracle.steps(orc.make_params(N, nf, **kw), s0, 1)
    return N, nf, kw, modes, s0, want


def test_one_step_bit_exact_every_way(case):
    import torch

    N, nf, kw, modes, s0, want = case
    p = asd.Params.make(N, nf, **kw)
    with asd.Context(p, modes=["fp64"]) as ctx:
        for kern in ("fused", "stages", "auto"):
            ctx.set_llg_kernel(kern)
            ctx.set_spins(s0, as_origin=True)
            ctx.step(1)
            assert np.array_equal(ctx.get_spins(), want), kern
        ctx.set_llg_kernel("auto")
        buf = torch.from_numpy(s0.reshape(-1).copy()).pin_memory()
        ctx.step_host(buf.data_ptr(), buf.data_ptr(), "fp64")
        assert np.array_equal(buf.numpy().reshape(s0.shape), want), "step_host"
        buf.copy_(torch.from_numpy(s0.reshape(-1)))
        sq = torch.zeros(2, dtype=torch.float64).pin_memory()
        ctx.step_host_async(buf.data_ptr(), buf.data_ptr(), "fp64", sq.data_ptr())
        ctx.synchronize()
        assert np.array_equal(buf.numpy().reshape(s0.shape), want), "step_host_async"
    lens = np.linalg.norm(want, axis=-1)
    assert np.abs(lens - 1.0).max() < 1e-15


def test_step_commutes_with_translation_and_replica_permutation(case):
    N, nf, kw, modes, s0, want = case
    perm = np.random.default_rng(1).permutation(nf)
    with asd.Context(asd.Params.make(N, nf, **kw), modes=["fp64"]) as ctx:
        ctx.set_spins(roll(s0, N, 5, -17), as_origin=True)
        ctx.step(1)
        assert np.array_equal(ctx.get_spins(), roll(want, N, 5, -17))
        ctx.set_spins(np.ascontiguousarray(s0[perm]), as_origin=True)
        ctx.step(1)
        assert np.array_equal(ctx.get_spins(), want[perm])


def test_sqt_fp64_against_oracle_and_split_modes_within_tolerance(case, oracle):
    N, nf, kw, modes, s0, want = case
    ref = oracle.sqt_factorized(N, nf, N // 10, N // 10, want, s0)
    with asd.Context(asd.Params.make(N, nf, **kw), modes=modes) as ctx:
        ctx.set_spins(s0, as_origin=True)
        ctx.step(1)
        got = {m: ctx.sqt(m) for m in modes}
    assert abs(got["fp64"] - ref) <= 1e-12 * abs(ref)
    for m in modes:
        if m != "fp64":
            assert abs(got[m] - got["fp64"]) <= 1e-5 * abs(got["fp64"]), m


def test_more_tiles_than_a_32_bit_index(oracle):
    """N = 2900 (8.41 M sites): the split GEMM walks (M/128) x (M/256) =
    2.16e9 tiles, more than a 32-bit index holds.  Two replicas keep it to a
    few seconds.  One RK4 step bit for bit against the oracle; BF16x3 S(q,t)
    against the oracle's factorised FP64 value (1e-5 of |S| plus 4 times the
    operands' precision floor 2^-17 sqrt(K) / (3 nfile)); the FP64 path, one
    block per 128 x 128 tile (4.3e9 blocks), refuses with ASD_ERR_UNSUPPORTED.
    About 90 s on a B200: K = 6 pads to one k block of 64, so the GEMM is
    bound by streaming its operands, not by the tensor cores."""
    N, nf = 2900, 2
    kw = dict(J1=1.0, alpha=0.05, h=(0.0, 0.0, 0.3), dt=0.01)
    s0 = asd.random_spins(N, nf, seed=29)
    with asd.Context(asd.Params.make(N, nf, **kw), modes=["fp64", "bf16x3"]) as ctx:
        ctx.set_spins(s0, as_origin=True)
        ctx.step(1)
        st = ctx.get_spins()
        assert np.array_equal(st, oracle.steps(orc.make_params(N, nf, **kw), s0, 1))
        got = ctx.sqt("bf16x3")
        with pytest.raises(asd.AsdError) as e:
            ctx.sqt("fp64")
        assert e.value.code == asd.ASD_ERR_UNSUPPORTED
    want = oracle.sqt_factorized(N, nf, N // 10, N // 10, st, s0)
    floor = 2.0 ** -17 * (3 * nf) ** 0.5 / (3 * nf)
    assert abs(got - want) <= 1e-5 * abs(want) + 4 * floor, (got, want)


def test_known_answers_at_full_size():
    """At 256 x 256 x 1000 with the headline model (J = 1, J2 = -0.3, alpha =
    0.02): a uniform ferromagnet, every spin along z, is stationary (H is
    parallel to S, the torque is exactly zero) through both LLG kernels, bit
    for bit; with every replica the same configuration the connected S(q,t)
    vanishes (C_ij = m_i . z_j), here through the FP64 path."""
    N, nf = 256, 1000
    kw = dict(J1=1.0, J2=-0.3, alpha=0.02, dt=0.005)
    up = np.zeros((nf, N * N, 3))
    up[..., 2] = 1.0
    with asd.Context(asd.Params.make(N, nf, **kw), modes=["fp64"]) as ctx:
        for kern in ("fused", "stages"):
            ctx.set_llg_kernel(kern)
            ctx.set_spins(up, as_origin=True)
            ctx.step(3)
            assert np.array_equal(ctx.get_spins(), up), kern
        del up
        same = np.repeat(asd.random_spins(N, 1, seed=7), nf, axis=0)
        ctx.set_llg_kernel("auto")
        ctx.set_spins(same, as_origin=True)
        ctx.step(2)
        assert abs(ctx.sqt("fp64")) < 1e-9
