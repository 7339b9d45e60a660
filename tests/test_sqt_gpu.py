"""GPU parity of S(q,t) (through the C ABI) against the oracle and the
reference fixtures.

Tolerances: FP64 paths 1e-12 relative; the split-precision tensor-core paths
(TF32x3, BF16x3, FP16x3) 1e-5 relative, the bound the design targets."""
from __future__ import annotations

import numpy as np
import pytest

import asd_b200 as asd
import oracle as orc
from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "tf32x3": 1e-5, "bf16x3": 1e-5, "fp16x3": 1e-5}


@pytest.mark.parametrize("name", ["llg_n12_f4", "llg_n20_f6"])
def test_sqt_matches_reference_fixture(golden, name):
    g = golden(name)
    N, nf = int(g["N"]), int(g["nfile"])
    ref = complex(g["sqt_gemm_len1"])
    with asd.Context(asd.Params.make(N, nf, J1=float(g["J1"]), dt=float(g["dt"]))) as ctx:
        ctx.set_spins(g["spins0"], as_origin=True)
        ctx.step(int(g["nsteps"]))
        assert np.array_equal(ctx.get_spins(), g["steps_len1"])
        for mode, tol in TOL.items():
            got = ctx.sqt(mode)
            assert rel_err(got, ref) < tol, (mode, got, ref)


@pytest.mark.parametrize("N,nfile,steps", [(16, 8, 2), (32, 50, 3), (24, 200, 1), (40, 11, 4), (50, 64, 2)])
def test_sqt_modes_vs_oracle(oracle, N, nfile, steps):
    s0 = asd.random_spins(N, nfile, seed=N * 3 + nfile)
    kw = dict(J1=-1.0, alpha=0.05, h=(0.0, 0.0, 0.5), dt=0.005)
    with asd.Context(asd.Params.make(N, nfile, **kw)) as ctx:
        ctx.set_spins(s0, as_origin=True)
        ctx.step(steps)
        st = ctx.get_spins()
        vx = N // 10
        ref = oracle.sqt_factorized(N, nfile, vx, vx, st, s0)
        if N <= 32:
            assert rel_err(oracle.sqt_gemm(N, nfile, vx, vx, st, s0), ref) < 1e-12
        for mode, tol in TOL.items():
            got = ctx.sqt(mode)
            assert rel_err(got, ref) < tol, (mode, got, ref)


def test_sqt_at_origin_and_q_zero(oracle):
    """t = 0 (A = B) and q = 0 (vx = vy = 0, every phase 1)."""
    N, nf = 32, 40
    s0 = asd.random_spins(N, nf, seed=2)
    with asd.Context(asd.Params.make(N, nf, vx=0, vy=0)) as ctx:
        ctx.set_spins(s0, as_origin=True)
        ref = oracle.sqt_factorized(N, nf, 0, 0, s0, s0)
        for mode, tol in TOL.items():
            assert rel_err(ctx.sqt(mode), ref) < tol, mode


def test_sqt_repeatable_and_deterministic():
    N, nf = 48, 30
    s0 = asd.random_spins(N, nf, seed=7)
    with asd.Context(asd.Params.make(N, nf)) as ctx:
        ctx.set_spins(s0, as_origin=True)
        ctx.step(2)
        for mode in TOL:
            a = ctx.sqt(mode)
            b = ctx.sqt(mode)
            assert a == b, mode


@pytest.mark.parametrize("name", ["fused_dgemm_valid", "fused_dgemm_rows", "fused_dgemm_cols"])
def test_dropin_fused_dgemm_matches_reference(golden, name):
    g = golden(name)
    c = g["c_in"].copy()
    s = np.zeros(2 * 128)
    asd.fused_dgemm(int(g["m"]), int(g["n"]), int(g["k"]), float(g["alpha"]), g["a"],
                    int(g["lda"]), g["b"], int(g["ldb"]), c, int(g["ldc"]), g["q"], s)
    assert np.array_equal(c, g["c_out"])  # the same FMA chain per element
    total = np.array([s[0::2].sum(), s[1::2].sum()])
    assert np.allclose(total, g["sum"], rtol=1e-13, atol=1e-12)


def test_dropin_fused_dgemm_sqt_glue(oracle):
    """The reference's fused S(q,t) sequence (llg_sqt_fusion.c:370-441) run
    with the GPU fused_dgemm equals the oracle's fused form."""
    N, nf = 12, 6
    M, K = N * N, 3 * nf
    s0 = asd.random_spins(N, nf, seed=31)
    st = oracle.steps(orc.make_params(N, nf), s0, 3)
    ref = oracle.sqt_fused(N, nf, 1, 1, st, s0)
    a = np.ascontiguousarray(st.transpose(0, 2, 1).reshape(K, M))   # spint: A(j, 3i+c) at j + (3i+c)M
    b = np.ascontiguousarray(s0.transpose(1, 0, 2).reshape(M * K))   # spin_zero
    fint = st.mean(axis=0)
    zerot = s0.mean(axis=0)
    qx = 2 * np.pi * 1 / N
    r = np.arange(M) // N
    cc = np.arange(M) % N
    th = qx * (r[:, None] - r[None, :]) + qx * (cc[:, None] - cc[None, :])
    qm = np.exp(-1j * th)
    rows = (np.arange(M) // 4) * 8 + np.arange(M) % 4
    ldc = 2 * M
    qmat = np.zeros((M, ldc))  # [j][row]
    cmat = np.zeros((M, ldc))
    outer = fint @ zerot.T
    qmat[:, rows] = qm.real.T
    qmat[:, rows + 4] = qm.imag.T
    cmat[:, rows] = -(outer * qm.real).T
    cmat[:, rows + 4] = -(outer * qm.imag).T
    s = np.zeros(256)
    qf, cf = qmat.reshape(-1), cmat.reshape(-1).copy()
    asd.fused_dgemm(M, M, K, 1.0 / nf, a.reshape(-1), M, b, K, cf, ldc, qf, s)
    got = complex(s[0::2].sum(), s[1::2].sum()) / M
    assert rel_err(got, ref) < 1e-12


@pytest.mark.parametrize("pinned", [False, True])
def test_step_host_matches_the_device_path(pinned):
    """asd_ctx_step_host (host spins in, one step, spins and S(q,t) out, the
    read-back overlapped with the GEMM) equals set_spins + step + get_spins +
    sqt, also when the input and output buffers are the same."""
    import torch

    N, nf = 24, 10
    s0 = asd.random_spins(N, nf, seed=8)
    p = asd.Params.make(N, nf, J1=-1.0, alpha=0.05, h=(0, 0, 0.5), dt=0.005)
    with asd.Context(p) as a, asd.Context(p) as b:
        a.set_spins(s0, as_origin=True)
        b.set_spins(s0, as_origin=True)
        buf = torch.from_numpy(s0.reshape(-1).copy())
        if pinned:
            buf = buf.pin_memory()
        for step in range(3):
            got = a.step_host(buf.data_ptr(), buf.data_ptr(), "tf32x3")
            b.step(1)
            want = b.sqt("tf32x3")
            assert np.array_equal(buf.numpy().reshape(s0.shape), b.get_spins()), step
            assert got == want


@pytest.mark.parametrize("mode", ["tf32x3", "bf16x3", "fp16x3"])
@pytest.mark.parametrize("kernel", ["stages", "fused"])
def test_step_pipelined_behind_the_split_gemm(oracle, mode, kernel):
    """asd_ctx_step after a split-mode asd_ctx_sqt_async runs the next RK4 step
    beside that S(q,t)'s GEMM.  The pipelined sequence must give the same
    S(q,t) values and spins, bit for bit, as the fully ordered one (any other
    entry point in between, here asd_ctx_set_stream, orders them), and the
    spins must equal the oracle's FP64 trajectory."""
    import torch

    N, nf, n = 64, 48, 6
    s0 = asd.random_spins(N, nf, seed=21)
    p = asd.Params.make(N, nf, J1=-1.0, J2=0.1, alpha=0.05, h=(0, 0, 0.5), dt=0.005, vx=3, vy=1)
    stream = torch.cuda.current_stream()
    outs = []
    spins = []
    for ordered in (False, True):
        d = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
        with asd.Context(p, modes=[mode]) as ctx:
            ctx.set_llg_kernel(kernel)
            ctx.set_stream(stream.cuda_stream)
            ctx.set_spins(s0, as_origin=True)
            for i in range(n):
                if ordered:
                    ctx.set_stream(stream.cuda_stream)
                ctx.step(1)
                ctx.sqt_async(mode, d.data_ptr() + 16 * i)
            torch.cuda.synchronize()
            ctx.check_device_status()
            spins.append(ctx.get_spins())
        outs.append(d.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(spins[0], spins[1])
    want = oracle.steps(orc.make_params(N, nf, J1=-1.0, J2=0.1, alpha=0.05, h=(0, 0, 0.5),
                                        dt=0.005), s0, n)
    assert np.array_equal(spins[0], want)


@pytest.mark.parametrize("kernel,where", [("fused", "pinned"), ("stages", "pinned"),
                                          ("fused", "device")])
@pytest.mark.parametrize("nf", [200, 40, 7])
def test_step_host_async_consecutive_steps(oracle, nf, kernel, where):
    """asd_ctx_step_host_async: six steps enqueued back to back on one pinned
    buffer (each call's output is the next call's input, so every chunk's
    upload must wait for the previous call's download of that chunk), then
    one asd_ctx_synchronize.  200 replicas make chunks of 32 (six) and 8; 40
    make 32 + 8; 7 one chunk.  The spins equal the device path and the oracle
    bit for bit; each step's S(q,t) equals the device path's asd_ctx_sqt on
    the same state exactly (the same kernels in the same order).  The
    buffers may also be device memory."""
    import torch

    N = 16
    s0 = asd.random_spins(N, nf, seed=21)
    kw = dict(J1=-1.0, J2=0.2, alpha=0.05, h=(0, 0, 0.5), dt=0.005)
    p = asd.Params.make(N, nf, vx=3, vy=2, **kw)
    modes = ["tf32x3", "fp64", "bf16x3", "fp16x3", "fp64", "tf32x3"]
    with asd.Context(p) as a, asd.Context(p) as b:
        a.set_llg_kernel(kernel)
        a.set_spins(s0, as_origin=True)
        b.set_spins(s0, as_origin=True)
        buf = torch.from_numpy(s0.reshape(-1).copy())
        sq = torch.zeros(2 * len(modes), dtype=torch.float64)
        if where == "pinned":
            buf, sq = buf.pin_memory(), sq.pin_memory()
        else:
            buf, sq = buf.cuda(), sq.cuda()
        for i, mode in enumerate(modes):
            a.step_host_async(buf.data_ptr(), buf.data_ptr(), mode, sq.data_ptr() + 16 * i)
        a.synchronize()
        if where == "device":
            buf, sq = buf.cpu(), sq.cpu()
        want = s0
        for i, mode in enumerate(modes):
            b.step(1)
            assert complex(*sq[2 * i:2 * i + 2].tolist()) == b.sqt(mode), (i, mode)
            want = oracle.steps(orc.make_params(N, nf, **kw), want, 1)
        assert np.array_equal(buf.numpy().reshape(s0.shape), b.get_spins())
        assert np.array_equal(b.get_spins(), want)
        # the context keeps working synchronously afterwards
        buf = buf.pin_memory()
        got = a.step_host(buf.data_ptr(), buf.data_ptr(), "fp64")
        b.step(1)
        assert got == b.sqt("fp64")
        assert np.array_equal(buf.numpy().reshape(s0.shape), b.get_spins())


def test_step_host_async_needs_pinned_or_device_buffers():
    """Pageable host memory cannot be copied asynchronously: the call fails
    with ASD_ERR_INVALID before enqueueing anything."""
    import torch

    N, nf = 12, 4
    s0 = asd.random_spins(N, nf, seed=3)
    with asd.Context(asd.Params.make(N, nf, J1=1.0, dt=0.01), modes=["fp64"]) as a:
        a.set_spins(s0, as_origin=True)
        pageable = s0.reshape(-1).copy()
        sq = torch.zeros(2, dtype=torch.float64).pin_memory()
        with pytest.raises(asd.AsdError) as e:
            a.step_host_async(pageable.ctypes.data, pageable.ctypes.data, "fp64", sq.data_ptr())
        assert e.value.code == asd.ASD_ERR_INVALID
        assert np.array_equal(a.get_spins(), s0)


@pytest.mark.parametrize("kernel", ["fused", "stages"])
@pytest.mark.parametrize("nf,pinned", [(200, False), (200, True), (65, True), (128, True)])
def test_step_host_in_replica_chunks(oracle, nf, pinned, kernel):
    """Ensembles larger than one upload chunk (64 replicas and up) take the
    pipelined asd_ctx_step_host: per replica chunk, upload, RK4 (the one-launch
    step into the other state buffer, or the four stage kernels in place),
    download and a GEMM over that chunk's K columns.  200 replicas make chunks of 64, 64,
    64 and a ragged 8 (65: 64 + 1; 128: two whole chunks).  The spins must
    equal the device path and the oracle
    bit for bit; S(q,t) must equal the device path exactly in the FP64 modes
    and agree to the split-precision tolerance (1e-5 of the FP64 value) in
    the split modes, whose partial sums are added in another order."""
    import torch

    N = 16
    s0 = asd.random_spins(N, nf, seed=12)
    kw = dict(J1=-1.0, J2=0.2, alpha=0.05, h=(0, 0, 0.5), dt=0.005)
    p = asd.Params.make(N, nf, vx=3, vy=2, **kw)
    with asd.Context(p) as a, asd.Context(p) as b:
        a.set_llg_kernel(kernel)
        a.set_spins(s0, as_origin=True)
        b.set_spins(s0, as_origin=True)
        buf = torch.from_numpy(s0.reshape(-1).copy())
        if pinned:
            buf = buf.pin_memory()
        want_spins = s0
        for step, mode in enumerate(["tf32x3", "fp64", "bf16x3", "fp16x3", "fp64", "tf32x3"]):
            got = a.step_host(buf.data_ptr(), buf.data_ptr(), mode)
            b.step(1)
            ref = b.sqt("fp64")
            want_spins = oracle.steps(orc.make_params(N, nf, **kw), want_spins, 1)
            assert np.array_equal(buf.numpy().reshape(s0.shape), b.get_spins()), step
            assert np.array_equal(b.get_spins(), want_spins), step
            if mode.startswith("fp64"):
                assert got == b.sqt(mode), (step, mode)
            else:
                # each split result within 1e-5 of FP64; the chunked one sums
                # shorter K ranges in FP32 and is usually the closer of the two
                assert abs(got - ref) <= 1e-5 * abs(ref), (step, mode, got, ref)
                assert abs(b.sqt(mode) - ref) <= 1e-5 * abs(ref), (step, mode)


@pytest.mark.parametrize("spin_len", [1e-3, 1.5, 3e4])
def test_fp16x3_scale_follows_spin_len(oracle, spin_len):
    """FP16x3 scales the spins by a power of two (spin_len * scale in
    [2^12, 2^13)) before the split, so spins of any length keep the FP16
    pair's 22 bits: 1e-3 would leave the lo parts subnormal and 3e4 would
    come close to FP16's largest value without it.  A change of spin_len
    through asd_ctx_set_params changes the scale, and the origin is split
    again with it.  A component beyond FP16's range after scaling gives a
    non-finite S(q,t), not a wrong finite one.  The exchange torque grows as
    spin_len^2, so dt = 0.005 / spin_len keeps the same dynamics at every
    length (without a field, which would not scale)."""
    N, nf = 32, 40
    kw = dict(J1=-1.0, alpha=0.05, dt=0.005 / spin_len)
    s0 = asd.random_spins(N, nf, seed=5, spin_len=spin_len)
    p = asd.Params.make(N, nf, spin_len=spin_len, **kw)
    with asd.Context(p, modes=["fp64", "fp16x3"]) as ctx:
        ctx.set_spins(s0, as_origin=True)
        ctx.step(3)
        st = ctx.get_spins()
        ref = oracle.sqt_factorized(N, nf, N // 10, N // 10, st, s0)
        assert rel_err(ctx.sqt("fp16x3"), ref) < 1e-5
        assert rel_err(ctx.sqt("fp64"), ref) < 1e-12
        # a new length: the next step renormalises to it, the origin keeps the
        # old one, and both operands take the new scale
        ctx.set_params(asd.Params.make(N, nf, spin_len=spin_len * 300.0, **kw))
        ctx.step(1)
        ref = ctx.sqt("fp64")
        assert rel_err(ctx.sqt("fp16x3"), ref) < 1e-5
    big = s0.copy()
    big[0, 0, 0] = spin_len * 2.0 ** 5  # at least 2^17 > 65504 after scaling
    with asd.Context(p, modes=["fp16x3"]) as ctx:
        ctx.set_spins(big, as_origin=True)
        assert not np.isfinite(ctx.sqt("fp16x3"))
