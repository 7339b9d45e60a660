"""The plain FP64 S(q,t) path: the FP64 tensor-core GEMM (mma.sync m16n8k8
.f64) with its fused epilogue, against the oracle.

* The fragment layout the GEMM assumes, checked on one MMA against a host
  product.
* S(q,t) at one q within 1e-12 of the oracle's factorised FP64 value, for even
  K (16-byte copies) and odd K (8-byte copies), lattices whose site count is
  not a multiple of the 128-site tile, and repeated calls bit for bit.
* The q grid through the diagonal partials, every mode, at N = 100, 128 and
  136, on a sample of q against the oracle's factorised value at that q, and
  two runs bit for bit.
* The measured FP64 peaks the benchmark quotes are plausible."""
from __future__ import annotations

import numpy as np
import pytest

import asd_b200 as asd
from conftest import rel_err

pytestmark = pytest.mark.gpu


def test_dmma_fragment_layout():
    import torch

    g = torch.Generator().manual_seed(7)
    A = torch.randn(16, 8, dtype=torch.float64, generator=g)
    B = torch.randn(8, 8, dtype=torch.float64, generator=g)
    dA, dB = A.cuda(), B.cuda()
    dD = torch.full((16, 8), float("nan"), dtype=torch.float64, device="cuda")
    asd.check_dmma_layout(dA.data_ptr(), dB.data_ptr(), dD.data_ptr(),
                          torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    want = A @ B
    assert torch.allclose(dD.cpu(), want, rtol=1e-13, atol=1e-13), (dD.cpu() - want).abs().max()


@pytest.mark.parametrize("which", ["fma", "dmma"])
def test_fp64_peak_is_plausible(which):
    tf, ms = asd.measure_fp64_peak(which)
    assert ms > 0.0
    assert 5.0 < tf < 200.0, tf


@pytest.mark.parametrize("N,nfile,steps", [(20, 8, 2), (20, 7, 2), (37, 33, 1), (12, 3, 3),
                                           (24, 40, 1)])
def test_fp64_sqt_vs_oracle(oracle, N, nfile, steps):
    """K = 3 nfile even (24, 120) and odd (21, 99, 9); N*N = 400, 1369, 144,
    576 sites: every lattice has a partial tile."""
    s0 = asd.random_spins(N, nfile, seed=N * 31 + nfile)
    kw = dict(J1=-1.0, J2=0.2, alpha=0.05, h=(0.0, 0.0, 0.5), dt=0.005)
    vx, vy = max(1, N // 10), max(1, N // 7)
    with asd.Context(asd.Params.make(N, nfile, vx=vx, vy=vy, **kw), modes=["fp64"]) as ctx:
        ctx.set_spins(s0, as_origin=True)
        ctx.step(steps)
        st = ctx.get_spins()
        a = ctx.sqt("fp64")
        b = ctx.sqt("fp64")
    want = oracle.sqt_factorized(N, nfile, vx, vy, st, s0)
    assert rel_err(a, want) < 1e-12, (a, want)
    assert a == b


def test_fp64_single_replica_is_zero():
    """With one replica the connected part is identically zero (m_i = S_i):
    the FP64 path gives zero up to rounding of the O(1) terms it cancels."""
    N = 12
    s0 = asd.random_spins(N, 1, seed=5)
    with asd.Context(asd.Params.make(N, 1, J1=1.0, dt=0.01), modes=["fp64"]) as ctx:
        ctx.set_spins(s0, as_origin=True)
        ctx.step(3)
        v = ctx.sqt("fp64")
        mag = ctx.sqt_magnitude()
    assert abs(v) < 1e-15
    assert mag < 1e-13


def test_fp64_kernel_is_timed():
    """asd_ctx_time_kernels records the FP64 GEMM launch and the RK4 step."""
    N, nf = 32, 10
    with asd.Context(asd.Params.make(N, nf, J1=1.0, dt=0.01), modes=["fp64"]) as ctx:
        ctx.set_spins(asd.random_spins(N, nf, seed=1), as_origin=True)
        ctx.time_kernels(True)
        ctx.step(3)
        ctx.sqt("fp64")
        ctx.sqt("fp64")
        ms_g, n_g = ctx.kernel_time("gemm")
        ms_l, n_l = ctx.kernel_time("llg")
        assert n_g == 2 and ms_g > 0.0
        assert n_l >= 3 and ms_l > 0.0
        assert ctx.kernel_time("gemm") == (0.0, 0)  # read once
        ctx.time_kernels(False)
        ctx.sqt("fp64")
        assert ctx.kernel_time("gemm") == (0.0, 0)


@pytest.mark.parametrize("N,nfile", [(100, 6), (128, 12), (136, 5)])
def test_qgrid_large_lattices(oracle, N, nfile):
    """N*N = 10000 (tiles span several lattice rows), 16384 (tiles are whole
    half rows) and 18496 sites, in every mode: sampled q against the oracle's
    factorised FP64 value at that q (FP64 1e-12, split modes 1e-5, of max |S|
    over the sample), and the grid twice, bit for bit."""
    s0 = asd.random_spins(N, nfile, seed=N + nfile)
    kw = dict(J1=1.0, alpha=0.1, dt=0.01)
    grids = {}
    with asd.Context(asd.Params.make(N, nfile, **kw)) as ctx:
        ctx.set_spins(s0, as_origin=True)
        ctx.step(2)
        st = ctx.get_spins()
        for mode in ("fp64", "tf32x3", "bf16x3", "fp16x3"):
            g1 = ctx.sqt_grid(mode)
            g2 = ctx.sqt_grid(mode)
            assert np.array_equal(g1, g2), mode
            grids[mode] = g1
    rng = np.random.default_rng(N)
    qs = [(0, 0), (N // 10, N // 10), (N - 1, 1), (1, N - 1), (N // 2, N // 3)]
    qs += [tuple(int(x) for x in rng.integers(0, N, size=2)) for _ in range(7)]
    want = {q: oracle.sqt_factorized(N, nfile, q[0], q[1], st, s0) for q in qs}
    scale = max(abs(v) for v in want.values())
    for mode, tol in (("fp64", 1e-12), ("tf32x3", 1e-5), ("bf16x3", 1e-5), ("fp16x3", 1e-5)):
        for q, w in want.items():
            assert abs(grids[mode][q] - w) <= tol * scale, (mode, q, grids[mode][q], w)
