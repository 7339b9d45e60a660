"""The cblas_dgemm drop-in on the GPU: every CBLAS layout and transpose
combination against numpy's FP64 product, the BLAS special cases, and the
reference's own gemm program (its S(q,t) sequence around cblas_dgemm,
gemm/llg_sqt_mkl.c:349-423, compiled from its sources into oracle/_ref)
running its GEMM through libasd_cblas.so.

Tolerance: the product is FP64 with FMA accumulation in another order than a
CPU BLAS, so |C - C_ref| <= 1e-13 (|alpha| |op(A)| |op(B)| + |beta| |C0|)
elementwise."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

import asd_b200 as asd
from conftest import ROOT

pytestmark = pytest.mark.gpu

R, CM, NT, T, H = 101, 102, 111, 112, 113
SHIM = asd.LIB_PATH.parent / "libasd_cblas.so"


def stored(x, order, ld, rows, cols):
    """The flat array BLAS reads for the rows x cols matrix x with leading
    dimension ld (column-major: ld >= rows; row-major: ld >= cols); padding
    holds a marker value."""
    if order == CM:
        buf = np.full((cols, ld), -7.25)
        buf[:, :rows] = x.T
    else:
        buf = np.full((rows, ld), -7.25)
        buf[:, :cols] = x
    return buf.reshape(-1).copy()


def loaded(buf, order, ld, rows, cols):
    if order == CM:
        return buf.reshape(cols, ld)[:, :rows].T
    return buf.reshape(rows, ld)[:, :cols]


@pytest.mark.parametrize("order", [CM, R])
@pytest.mark.parametrize("ta", [NT, T, H])
@pytest.mark.parametrize("tb", [NT, T])
@pytest.mark.parametrize("m,n,k", [(37, 29, 41), (130, 257, 64)])
def test_every_layout_against_numpy(order, ta, tb, m, n, k):
    rng = np.random.default_rng(m + 3 * n + 7 * k + ta + tb + order)
    opa = rng.standard_normal((m, k))
    opb = rng.standard_normal((k, n))
    c0 = rng.standard_normal((m, n))
    alpha, beta = 0.7, -1.3
    A = opa.T if ta != NT else opa  # the matrix as stored before op()
    B = opb.T if tb != NT else opb
    ra, ca = A.shape
    rb, cb = B.shape
    lda = (ra if order == CM else ca) + 3
    ldb = (rb if order == CM else cb) + 1
    ldc = (m if order == CM else n) + 2
    a, b, c = stored(A, order, lda, ra, ca), stored(B, order, ldb, rb, cb), stored(c0, order, ldc, m, n)
    pad = c.copy()
    asd.cblas_dgemm(order, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    got = loaded(c, order, ldc, m, n)
    want = alpha * (opa @ opb) + beta * c0
    scale = abs(alpha) * (np.abs(opa) @ np.abs(opb)) + abs(beta) * np.abs(c0)
    assert (np.abs(got - want) <= 1e-13 * scale).all()
    keep = np.ones_like(c, dtype=bool)
    loaded(keep, order, ldc, m, n)[...] = False
    assert np.array_equal(c[keep], pad[keep])  # the padding of C is untouched


def test_blas_special_cases():
    rng = np.random.default_rng(3)
    m, n, k = 20, 13, 9
    a = rng.standard_normal((k, m)).reshape(-1).copy()  # column-major m x k, lda = m
    b = rng.standard_normal((n, k)).reshape(-1).copy()  # column-major k x n, ldb = k
    A = a.reshape(k, m).T
    B = b.reshape(n, k).T
    # beta == 0: C is not read, NaN in it does not reach the result
    c = np.full(m * n, np.nan)
    asd.cblas_dgemm(CM, NT, NT, m, n, k, 2.0, a, m, b, k, 0.0, c, m)
    want = 2.0 * A @ B
    assert np.isfinite(c).all()
    assert np.allclose(c.reshape(n, m).T, want, rtol=1e-13, atol=1e-13)
    # alpha == 0: C = beta C exactly, A and B not read
    c0 = rng.standard_normal(m * n)
    c = c0.copy()
    asd.cblas_dgemm(CM, NT, NT, m, n, k, 0.0, None, m, None, k, -0.5, c, m)
    assert np.array_equal(c, -0.5 * c0)
    # k == 0: the same
    c = c0.copy()
    asd.cblas_dgemm(CM, NT, NT, m, n, 0, 1.0, None, m, None, 1, 3.0, c, m)
    assert np.array_equal(c, 3.0 * c0)
    # alpha == 0 and beta == 0: zeros, also over NaN
    c = np.full(m * n, np.nan)
    asd.cblas_dgemm(CM, NT, NT, m, n, k, 0.0, None, m, None, k, 0.0, c, m)
    assert (c == 0.0).all()
    # two calls in a row reuse the cached device buffers with other shapes
    c = np.zeros(3 * 2)
    asd.cblas_dgemm(R, NT, NT, 3, 2, 1, 1.0, np.array([1.0, 2.0, 3.0]), 1, np.array([4.0, 5.0]),
                    2, 0.0, c, 2)
    assert np.array_equal(c, np.array([4.0, 5.0, 8.0, 10.0, 12.0, 15.0]))


def test_correlation_gemm_shape():
    """The reference's call (gemm/llg_sqt_mkl.c:378): column-major, no
    transposes, C (M x M) = (1/nfile) A (M x K) B (K x M), lda = ldc = M,
    ldb = K, beta = 0, at M = 4096 sites and K = 3 * 100."""
    rng = np.random.default_rng(5)
    M, K = 4096, 300
    a = rng.uniform(-1, 1, M * K)
    b = rng.uniform(-1, 1, K * M)
    c = np.empty(M * M)
    asd.cblas_dgemm(CM, NT, NT, M, M, K, 0.01, a, M, b, K, 0.0, c, M)
    A = a.reshape(K, M).T
    B = b.reshape(M, K).T
    want = 0.01 * (A @ B)
    scale = 0.01 * (np.abs(A) @ np.abs(B))
    assert (np.abs(c.reshape(M, M).T - want) <= 1e-13 * scale).all()


@pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "libref_gemm.so").exists(),
                    reason="the reference's gemm program is not built")
def test_reference_gemm_program_runs_through_the_shim():
    """The reference's gemm program code (libref_gemm.so, linked against a CPU
    OpenBLAS) with libasd_cblas.so loaded ahead of it: its cblas_dgemm calls
    land on the GPU, and its S(q,t) equals the oracle's restatement of the same
    sequence.  A child process, so that no other BLAS is loaded before."""
    code = f"""
import ctypes as C, sys
sys.path.insert(0, {str(ROOT / 'oracle')!r})
shim = C.CDLL({str(SHIM)!r}, mode=C.RTLD_GLOBAL)
shim.asd_cblas_calls.restype = C.c_long
import oracle as orc
N, nf = 20, 6
s0 = orc.random_spins(N, nf, seed=9)
o = orc.Oracle()
st = o.steps(orc.make_params(N, nf), s0, 3)
ref = orc.RefLib("gemm")
ref.setup(N, nf, threads=2)
got = ref.gemm_sqt(st, s0)
want = o.sqt_gemm(N, nf, N // 10, N // 10, st, s0)
print(shim.asd_cblas_calls(), abs(got - want) / abs(want))
"""
    r = subprocess.run(["python", "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    calls, err = r.stdout.split()
    assert int(calls) >= 1  # the reference's GEMM reached the GPU
    assert float(err) < 1e-12
