"""The cblas_dgemm drop-in without a GPU: libasd_cblas.so exports exactly what
include/asd_cblas.h declares, and asd_cblas_dgemm checks its arguments the
way BLAS does (gemm/llg_sqt_mkl.c:378 is the reference's call) before it
touches a device; the calls that BLAS defines as doing nothing return at
once."""
from __future__ import annotations

import ctypes as C
import re
import subprocess

import numpy as np
import pytest

import asd_b200 as asd
from conftest import ROOT

SHIM = asd.LIB_PATH.parent / "libasd_cblas.so"
HEADER = ROOT / "include" / "asd_cblas.h"
R, Cm, N, T, H = 101, 102, 111, 112, 113


def test_shim_exports_every_declared_symbol():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    decl = set(re.findall(r"^\s*(?:void|long)\s+([A-Za-z_]\w*)\s*\(", text, flags=re.M))
    assert decl == {"cblas_dgemm", "asd_cblas_calls"}
    out = subprocess.run(["nm", "-D", "--defined-only", str(SHIM)], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert exported == decl


@pytest.mark.parametrize("args", [
    (5, N, N, 2, 2, 2, 2, 2, 2),      # order
    (Cm, 7, N, 2, 2, 2, 2, 2, 2),     # transa
    (Cm, N, 0, 2, 2, 2, 2, 2, 2),     # transb
    (Cm, N, N, -1, 2, 2, 2, 2, 2),    # m < 0
    (Cm, N, N, 4, 2, 3, 3, 3, 4),     # lda < m (column-major, no transpose)
    (Cm, T, N, 4, 2, 3, 2, 3, 4),     # lda < k (A transposed)
    (Cm, N, N, 4, 2, 3, 4, 2, 4),     # ldb < k
    (Cm, N, T, 4, 2, 3, 4, 1, 4),     # ldb < n (B transposed)
    (Cm, N, N, 4, 2, 3, 4, 3, 3),     # ldc < m
    (R, N, N, 4, 2, 3, 2, 2, 2),      # row major: lda < k
    (R, N, N, 4, 2, 3, 3, 1, 2),      # row major: ldb < n
    (R, N, N, 4, 2, 3, 3, 2, 1),      # row major: ldc < n
])
def test_invalid_arguments_are_rejected(args):
    order, ta, tb, m, n, k, lda, ldb, ldc = args
    a = np.ones(64)
    b = np.ones(64)
    c = np.full(64, 3.0)
    rc = asd.load().asd_cblas_dgemm(order, ta, tb, m, n, k, 1.0, C.c_void_p(a.ctypes.data), lda,
                                    C.c_void_p(b.ctypes.data), ldb, 0.0,
                                    C.c_void_p(c.ctypes.data), ldc)
    assert rc == asd.ASD_ERR_INVALID, asd.last_error()
    assert (c == 3.0).all()


def test_calls_that_do_nothing_return_without_a_device():
    c = np.full(12, 3.0)
    lib = asd.load()
    p = C.c_void_p(c.ctypes.data)
    # m == 0, n == 0: nothing to compute (NULL A and B are fine then)
    assert lib.asd_cblas_dgemm(Cm, N, N, 0, 3, 4, 1.0, None, 1, None, 4, 2.0, p, 1) == asd.ASD_OK
    assert lib.asd_cblas_dgemm(R, T, H, 3, 0, 4, 1.0, None, 3, None, 4, 2.0, p, 1) == asd.ASD_OK
    # alpha == 0 or k == 0 with beta == 1: C stays as it is
    assert lib.asd_cblas_dgemm(Cm, N, N, 3, 4, 0, 1.0, None, 3, None, 1, 1.0, p, 3) == asd.ASD_OK
    assert lib.asd_cblas_dgemm(Cm, N, N, 3, 4, 2, 0.0, None, 3, None, 2, 1.0, p, 3) == asd.ASD_OK
    assert (c == 3.0).all()


def test_shim_reports_and_counts_its_calls():
    """The shim forwards to asd_cblas_dgemm, prints BLAS-style errors on
    stderr and counts its calls (here in a child process of its own)."""
    code = (
        "import ctypes as C, numpy as np\n"
        f"s = C.CDLL({str(SHIM)!r})\n"
        "s.asd_cblas_calls.restype = C.c_long\n"
        "c = np.full(4, 3.0)\n"
        "s.cblas_dgemm.argtypes = [C.c_int]*6 + [C.c_double, C.c_void_p, C.c_int, C.c_void_p,"
        " C.c_int, C.c_double, C.c_void_p, C.c_int]\n"
        "s.cblas_dgemm(102, 111, 111, 2, 2, 2, 1.0, None, 1, None, 2, 0.0,"
        " C.c_void_p(c.ctypes.data), 2)\n"
        "s.cblas_dgemm(102, 111, 111, 0, 2, 2, 1.0, None, 1, None, 2, 0.0,"
        " C.c_void_p(c.ctypes.data), 2)\n"
        "print(s.asd_cblas_calls(), float(c.sum()))\n")
    r = subprocess.run(["python", "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.split() == ["2", "12.0"]
    assert "libasd_cblas cblas_dgemm:" in r.stderr and "leading dimension" in r.stderr
