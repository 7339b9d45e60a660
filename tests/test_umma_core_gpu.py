"""The tcgen05 core of the split S(q,t) GEMM on its own: the raw FP32
accumulator (asd_umma_gemm_f32) against an FP64 product of the same split
operands computed by torch.  This isolates descriptor, swizzle and TMEM
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
    else:
        hi = tf32_round(x)
        lo = tf32_round(x - hi.double())
    return hi.contiguous(), lo.contiguous()


@pytest.mark.parametrize("kind,rows,Kp,chunk", [(1, 256, 32, 0), (2, 256, 64, 0), (1, 512, 96, 0),
                                                (2, 768, 192, 0), (1, 1024, 1504, 0),
                                                (2, 512, 1536, 0), (1, 1024, 1504, 256),
                                                (2, 512, 1536, 512), (2, 256, 640, 64)])
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
    # lo*lo term and the representation error of hi+lo, plus the accumulation
    exact = A @ B.T
    split_eps = 2.0 ** -15 if kind == 2 else 2.0 ** -20
    bound = (split_eps + max(2e-6, steps * 2.0 ** -24)) * scale
    assert (C.double() - exact).abs().max().item() <= bound


def test_cta_pair_kernel_matches():
    """The CTA-pair form of the GEMM (cta_group::2, M = 256 over two SMs,
    selected by ASD_UMMA_PAIR=1, read once per process), checked in a child
    process: the raw product on several shapes against the same bound as
    above, and S(q,t) through a context against the FP64 path."""
    import os
    import subprocess
    import sys

    code = (
        "import sys; sys.path[:0] = {paths!r}\n"
        "import test_umma_core_gpu as t\n"
        "for case in ((1, 256, 32, 0), (2, 768, 192, 0), (1, 1024, 1504, 256),\n"
        "             (2, 512, 1536, 512)):\n"
        "    t.test_umma_core_matches_fp64_product(*case)\n"
        "import asd_b200 as asd\n"
        "p = asd.Params.make(40, 12, J1=-1.0, alpha=0.05, h=(0, 0, 0.5), dt=0.005, vx=2, vy=1)\n"
        "with asd.Context(p) as c:\n"
        "    c.set_spins(asd.random_spins(40, 12, seed=3), as_origin=True)\n"
        "    c.step(4)\n"
        "    ref = c.sqt('fp64')\n"
        "    for m in ('tf32x3', 'bf16x3'):\n"
        "        assert abs(c.sqt(m) - ref) <= 1e-5 * abs(ref), m\n"
        "print('ok')\n"
    ).format(paths=[os.path.dirname(__file__)] + sys.path)
    env = dict(os.environ, ASD_UMMA_PAIR="1")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stderr[-2000:]


@pytest.mark.parametrize("group", [7, 64])
def test_raster_group_size_changes_only_the_tile_order(group):
    """ASD_UMMA_GROUP_M (row tiles per raster group, read once per process)
    only reorders the tiles, so in a child process every product element
    still meets the bound above.  2048 rows give 16 row tiles, i.e. groups of
    7, 7 and 2, or one group smaller than 64.  S(q,t) through a context
    (1792 padded rows, 14 row tiles) stays within 1e-5 of the FP64 path."""
    import os
    import subprocess
    import sys

    code = (
        "import sys; sys.path[:0] = {paths!r}\n"
        "import test_umma_core_gpu as t\n"
        "for case in ((1, 2048, 64, 0), (2, 2048, 128, 0)):\n"
        "    t.test_umma_core_matches_fp64_product(*case)\n"
        "import asd_b200 as asd\n"
        "p = asd.Params.make(40, 12, J1=-1.0, alpha=0.05, h=(0, 0, 0.5), dt=0.005, vx=2, vy=1)\n"
        "with asd.Context(p) as c:\n"
        "    c.set_spins(asd.random_spins(40, 12, seed=3), as_origin=True)\n"
        "    c.step(4)\n"
        "    ref = c.sqt('fp64')\n"
        "    for m in ('tf32x3', 'bf16x3'):\n"
        "        assert abs(c.sqt(m) - ref) <= 1e-5 * abs(ref), m\n"
        "print('ok')\n"
    ).format(paths=[os.path.dirname(__file__)] + sys.path)
    env = dict(os.environ, ASD_UMMA_GROUP_M=str(group))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stderr[-2000:]
