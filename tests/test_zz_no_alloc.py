"""asd_sqt_split_noalloc: S(q,t) through the split tensor-core GEMM without
any allocation, for callers that must not call cudaMalloc/cudaFree while they
step (their device memory belongs to their own pool with a fixed budget, or
an allocation call would synchronise the device inside their step loop).

The test builds the entry point's inputs itself (split operands and epilogue
vectors, with torch), calls it twice in a row through the C ABI and compares
both results with the context API's S(q,t) for the same spins and with the
oracle's FP64 value, within the split modes' tolerance.  After a first call
(which may load the library's device code), further calls must leave both
torch's allocator and the device's free memory unchanged.  It sits in its own
file, collected last."""
from __future__ import annotations

import math

import numpy as np
import pytest

import asd_b200 as asd
from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-5  # the split modes' tolerance in tests/test_sqt_gpu.py


def tf32_round(x):
    import torch

    i = x.float().contiguous().view(torch.int32)
    i = (i + 0x1000) & ~0x1FFF  # round to nearest, ties away from zero
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


def inputs(torch, spins_t, spins_0, N, nfile, kind, vx):
    M, K = N * N, 3 * nfile
    rows = (M + 255) // 256 * 256
    ke = 64 if kind == 2 else 32
    Kp = (K + ke - 1) // ke * ke

    def operand(s):
        a = np.zeros((rows, Kp))
        a[:M, :K] = np.ascontiguousarray(s.transpose(1, 0, 2)).reshape(M, K)  # [site][replica*3+c]
        return split(torch.from_numpy(a).cuda(), kind)

    ah, al = operand(spins_t)
    bh, bl = operand(spins_0)
    q = 2.0 * math.pi * vx / N
    site = np.arange(M)
    th = q * (site // N) + q * (site % N)
    row4 = np.zeros((rows, 4), np.float32)
    row1 = np.zeros(rows, np.float32)
    col4 = np.zeros((rows, 4), np.float32)
    col1 = np.zeros(rows, np.float32)
    row4[:M, :3] = spins_t.mean(axis=0)
    row4[:M, 3] = np.cos(th)
    row1[:M] = -np.sin(th)
    col4[:M, :3] = spins_0.mean(axis=0)
    col4[:M, 3] = np.cos(th)
    col1[:M] = np.sin(th)
    vecs = [torch.from_numpy(v).cuda() for v in (row4, row1, col4, col1)]
    return rows, Kp, (ah, al, bh, bl), vecs


@pytest.mark.parametrize("mode,kind", [("bf16x3", 2), ("tf32x3", 1)])
def test_noalloc_matches_context_api(mode, kind, oracle):
    import torch

    N, nfile = 32, 40
    s0 = asd.random_spins(N, nfile, seed=17)
    with asd.Context(asd.Params.make(N, nfile, J1=1.0, alpha=0.05, dt=0.01)) as ctx:
        ctx.set_spins(s0, as_origin=True)
        ctx.step(3)
        st = ctx.get_spins()
        ref = ctx.sqt(mode)  # the existing entry point, default chunk of 512
    rows, Kp, ops, vecs = inputs(torch, st, s0, N, nfile, kind, N // 10)
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def call():
        out.fill_(float("nan"))
        asd.sqt_split_noalloc(kind, rows, Kp, *(t.data_ptr() for t in ops),
                              *(v.data_ptr() for v in vecs), 1.0 / nfile, 1.0 / (N * N), 512,
                              out.data_ptr(), stream)
        torch.cuda.synchronize()
        return complex(*out.tolist())

    call()  # the first call on this device may load the library's device code
    torch_bytes = torch.cuda.memory_allocated()
    free_bytes = torch.cuda.mem_get_info()[0]
    got = [call(), call()]  # two calls in a row share the fixed scratch
    assert torch.cuda.memory_allocated() == torch_bytes
    assert torch.cuda.mem_get_info()[0] == free_bytes
    want = oracle.sqt_factorized(N, nfile, N // 10, N // 10, st, s0)
    for g in got:
        assert rel_err(g, ref) < TOL, (g, ref)
        assert rel_err(g, want) < TOL, (g, want)
    assert got[0] == got[1]


def test_noalloc_rejects_bad_sizes():
    import torch

    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    buf = torch.zeros(256 * 64, dtype=torch.float32, device="cuda")
    p = buf.data_ptr()
    with pytest.raises(asd.AsdError) as e:
        asd.sqt_split_noalloc(2, 100, 64, p, p, p, p, p, p, p, p, 1.0, 1.0, 0, out.data_ptr())
    assert e.value.code == asd.ASD_ERR_INVALID
    with pytest.raises(asd.AsdError):
        asd.sqt_split_noalloc(3, 256, 64, p, p, p, p, p, p, p, p, 1.0, 1.0, 0, out.data_ptr())
