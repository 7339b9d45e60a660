"""The tcgen05 core of the split S(q,t) GEMM on its own, for TF32 (kind 1),
BF16 (kind 2) and FP16 (kind 3) operands: the raw FP32 accumulator
(asd_umma_gemm_f32) against an FP64 product of the same split operands
computed by torch.  This isolates descriptor, swizzle and TMEM
layout errors from the fused epilogue."""
from __future__ import annotations

import pytest

import asd_b200 as asd

pytestmark = pytest.mark.gpu


def tf32_round(x):
    import torch

    i = x.float().contiguous().view(torch.int32)
    i = (i + 0x1000) & ~0x1FFF  # round half away from zero on the magnitude bits
    return i.view(torch.float32)


def split(x, kind):
    import torch

    if kind == 2:
        hi = x.to(torch.bfloat16)
        lo = (x - hi.double()).to(torch.bfloat16)
    elif kind == 3:
        hi = x.to(torch.float16)
        lo = (x - hi.double()).to(torch.float16)
    else:
        hi = tf32_round(x)
        lo = tf32_round(x - hi.double())
    return hi.contiguous(), lo.contiguous()


@pytest.mark.parametrize("kind,rows,Kp,chunk", [(1, 256, 32, 0), (2, 256, 64, 0), (1, 512, 96, 0),
                                                (2, 768, 192, 0), (1, 1024, 1504, 0),
                                                (2, 512, 1536, 0), (1, 1024, 1504, 256),
                                                (2, 512, 1536, 512), (2, 256, 640, 64),
                                                (3, 256, 64, 0), (3, 768, 192, 0),
                                                (3, 512, 1536, 512)])
def test_umma_core_matches_fp64_product(kind, rows, Kp, chunk):
    import torch

    g = torch.Generator(device="cuda").manual_seed(rows + Kp + kind)
    A = torch.randn(rows, Kp, dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn(rows, Kp, dtype=torch.float64, device="cuda", generator=g) * 0.5 + 0.1
    ah, al = split(A, kind)
    bh, bl = split(B, kind)
    C = torch.full((rows, rows), float("nan"), dtype=torch.float32, device="cuda")
    asd.umma_gemm_f32(kind, rows, Kp, ah.data_ptr(), al.data_ptr(), bh.data_ptr(), bl.data_ptr(),
                      C.data_ptr(), rows, chunk, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    Ah, Al, Bh, Bl = (t.double() for t in (ah, al, bh, bl))
    ref = Ah @ Bh.T + Ah @ Bl.T + Al @ Bh.T
    err = (C.double() - ref).abs().max().item()
    scale = (Ah.abs() @ Bh.abs().T).max().item()
    assert not torch.isnan(C).any()
    # the tensor cores' FP32 accumulation: error grows with the number of
    # accumulation steps in one chunk (3 products per K step of 8 or 16)
    steps = 3 * (chunk or Kp) / (8 if kind == 1 else 16)
    assert err <= max(2e-6, steps * 2.0 ** -24) * scale, (err, scale)
    # and the split product is close to the exact FP64 product: the dropped
    # lo*lo term and the representation error of hi+lo (FP16 keeps TF32's
    # 11-bit significand; its lo parts of |x| < 1/4 are subnormal, an absolute
    # error of at most 2^-25), plus the accumulation
    exact = A @ B.T
    split_eps = 2.0 ** -15 if kind == 2 else 2.0 ** -20
    bound = (split_eps + max(2e-6, steps * 2.0 ** -24)) * scale
    assert (C.double() - exact).abs().max().item() <= bound


@pytest.mark.parametrize("kind,rows,Kp", [(1, 2560, 64), (2, 2560, 128), (2, 4096, 64),
                                          (3, 2560, 128)])
def test_partial_raster_group(kind, rows, Kp):
    """Tiles are walked in raster groups of 16 row tiles.  2560 rows give 20
    row tiles (one group of 16, then a partial group of 4) and 4096 rows give
    32 (two whole groups): every product element still meets the bound of the
    test above, so the raster only reorders the tiles."""
    test_umma_core_matches_fp64_product(kind, rows, Kp, 0)


def test_partial_raster_group_sqt():
    """S(q,t) through a context whose padded rows (1792 = 14 row tiles) form
    one partial raster group stays within 1e-5 of the FP64 path."""
    p = asd.Params.make(40, 12, J1=-1.0, alpha=0.05, h=(0, 0, 0.5), dt=0.005, vx=2, vy=1)
    with asd.Context(p) as c:
        c.set_spins(asd.random_spins(40, 12, seed=3), as_origin=True)
        c.step(4)
        ref = c.sqt("fp64")
        for m in ("tf32x3", "bf16x3", "fp16x3"):
            assert abs(c.sqt(m) - ref) <= 1e-5 * abs(ref), m
