"""Failure paths and uninitialised reads of the context API, on the GPU.

* Allocation failures are injected on the host (asd_debug_fail_alloc): the
  n-th device allocation of the context API fails as cudaMalloc does on a
  full device.  Each failure must come back as ASD_ERR_NOMEM, hand out no
  context, keep no device memory, and leave the context it happened in
  usable.  The reference checks no allocation at all (llg_sqt_baseline.c
  mallocs without a test); no GPU fault is involved here.
* Scratch poisoning (asd_ctx_debug_poison): NaN bytes in every buffer that
  carries nothing from one call to the next, before every call of a sequence
  that runs every kernel of the context API.  A kernel that read such a
  buffer before writing it would give NaN or other numbers; the results must
  equal an unpoisoned context's bit for bit (S(q,t) on the q grid within the
  run-to-run variation of its atomic bin sums).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import asd_b200 as asd

pytestmark = pytest.mark.gpu

KW = dict(J1=-1.0, J2=0.1, alpha=0.05, h=(0.0, 0.0, 0.5), dt=0.005)


def test_create_allocation_failures_leak_nothing():
    import torch

    # 25 MB per state array, so that a leaked array shows in cudaMemGetInfo
    p = asd.Params.make(128, 64, **KW)
    lib = asd.load()
    with asd.Context(p):  # loads the modules and cuBLAS once
        pass
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    failed = 0
    try:
        for n in range(1, 100):
            asd.debug_fail_alloc(n)
            h = C.c_void_p()
            rc = lib.asd_ctx_create(C.byref(p), 0, C.byref(h))
            if rc == asd.ASD_OK:
                assert lib.asd_ctx_destroy(h) == asd.ASD_OK
                break
            assert rc == asd.ASD_ERR_NOMEM, (n, asd.last_error())
            assert "injected" in asd.last_error()
            assert not h.value
            failed += 1
        else:
            pytest.fail("asd_ctx_create never succeeded")
    finally:
        asd.debug_fail_alloc(0)
    assert failed >= 15  # every allocation of asd_ctx_create failed once
    free1 = torch.cuda.mem_get_info()[0]
    assert abs(free0 - free1) < (8 << 20), (free0, free1)


def _calls(s0, target):
    import torch

    def step_host(c):
        buf = torch.from_numpy(s0.reshape(-1).copy()).pin_memory()
        v = c.step_host(buf.data_ptr(), buf.data_ptr(), "tf32x3")
        return v, buf.numpy().copy()

    def step_host_async(c):
        buf = torch.from_numpy(s0.reshape(-1).copy()).pin_memory()
        sq = torch.zeros(2, dtype=torch.float64).pin_memory()
        c.step_host_async(buf.data_ptr(), buf.data_ptr(), "bf16x3", sq.data_ptr())
        c.synchronize()
        return tuple(sq.tolist()), buf.numpy().copy()

    return {
        "sqt_grid": lambda c: Grid(c.sqt_grid("fp64"), GRID_RTOL["fp64"]),
        "step_host": step_host,
        "step_host_async": step_host_async,
        "loss_grad": lambda c: c.loss_grad(8, 2, 3, target),
    }


class Grid:
    """S(q,t) on the q grid: its bins are summed with shared-memory atomics,
    so repeated runs agree to rtol of the largest value, not bit for bit."""

    def __init__(self, v, rtol):
        self.v, self.rtol = v, rtol

    def __eq__(self, other):
        return bool(np.isfinite(self.v).all() and np.isfinite(other.v).all() and
                    np.abs(self.v - other.v).max() <= self.rtol * np.abs(other.v).max())


GRID_RTOL = {"fp64": 1e-12, "tf32x3": 1e-6, "bf16x3": 1e-6, "fp16x3": 1e-6}


def _same(x, y):
    if isinstance(x, (tuple, list)):
        return len(x) == len(y) and all(_same(a, b) for a, b in zip(x, y))
    if isinstance(x, np.ndarray):
        return np.array_equal(x, y)
    return x == y


@pytest.mark.parametrize("call", ["sqt_grid", "step_host", "step_host_async", "loss_grad"])
def test_failed_work_space_allocation_leaves_the_context_usable(call):
    """The first call of each kind allocates its work space (72 replicas make
    the host-buffer steps work in replica chunks with their own staging).
    With the 1st, 2nd, ... of those allocations failing, the call returns
    ASD_ERR_NOMEM each time, until it makes fewer allocations than the
    injection counts and succeeds; then, with the spins set again, it gives
    what a context that never failed gives, bit for bit (the q grid
    included: its sums run in a fixed order)."""
    import torch

    N, nf = 16, 72
    s0 = asd.random_spins(N, nf, seed=31)
    target = np.array([0.3 + 0.1j, 0.2 - 0.05j, 0.1 + 0.0j, 0.05 + 0.02j])
    run = _calls(s0, target)[call]
    p = asd.Params.make(N, nf, **KW)
    with asd.Context(p) as a, asd.Context(p) as b:
        for c in (a, b):
            c.set_spins(s0, as_origin=True)
        failed = 0
        for n in range(1, 40):
            asd.debug_fail_alloc(n)
            try:
                got = run(a)
            except asd.AsdError as e:
                assert e.code == asd.ASD_ERR_NOMEM, (n, str(e))
                failed += 1
            else:
                break
            finally:
                asd.debug_fail_alloc(0)
                # work a failed call enqueued ends before its host buffers go
                torch.cuda.synchronize()
            a.set_spins(s0, as_origin=True)
        else:
            pytest.fail("the call never succeeded")
        assert failed >= 1
        assert _same(got, run(b))
        for c in (a, b):
            c.set_spins(s0, as_origin=True)
        assert _same(run(a), run(b))
        a.check_device_status()


@pytest.mark.parametrize("kernel", ["fused", "stages"])
def test_scratch_poisoning_changes_nothing(kernel):
    import torch

    N, nf = 32, 24
    s0 = asd.random_spins(N, nf, seed=32)
    target = np.array([0.3 + 0.1j, 0.2 - 0.05j, 0.1 + 0.0j])
    p = asd.Params.make(N, nf, vx=3, vy=1, **KW)

    def sequence(ctx, poison):
        def P():
            if poison:
                ctx.debug_poison()

        out = []
        ctx.set_llg_kernel(kernel)
        P()
        ctx.set_spins(s0, as_origin=True)
        for mode in ("fp64", "tf32x3", "bf16x3", "fp16x3"):
            P()
            ctx.step(1)
            P()
            out.append(ctx.sqt(mode))
        for mode in ("fp64", "tf32x3", "bf16x3", "fp16x3"):
            P()
            out.append(Grid(ctx.sqt_grid(mode), GRID_RTOL[mode]))
        P()
        cur = ctx.get_spins()
        buf = torch.from_numpy(cur.reshape(-1).copy()).pin_memory()
        P()
        out.append(ctx.step_host(buf.data_ptr(), buf.data_ptr(), "bf16x3"))
        out.append(buf.numpy().copy())
        sq = torch.zeros(4, dtype=torch.float64).pin_memory()
        for i, mode in enumerate(("tf32x3", "fp64")):
            P()
            ctx.step_host_async(buf.data_ptr(), buf.data_ptr(), mode, sq.data_ptr() + 16 * i)
            ctx.synchronize()
        out.append(sq.numpy().copy())
        out.append(buf.numpy().copy())
        P()
        ctx.set_spins(s0, as_origin=True)
        P()
        out.append(ctx.loss_grad(6, 2, 4, target))
        P()
        out.append(ctx.get_spins())
        ctx.check_device_status()
        return out

    with asd.Context(p) as a, asd.Context(p) as b:
        clean = sequence(a, False)
        poisoned = sequence(b, True)
    assert len(clean) == len(poisoned)
    for i, (x, y) in enumerate(zip(clean, poisoned)):
        assert _same(x, y), i  # NaN compares unequal, so no NaN got through
