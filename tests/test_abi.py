"""The C ABI boundary: libasd_b200.so loads, exports exactly what
include/asd_b200.h declares, and validates arguments before touching a GPU."""
from __future__ import annotations

import ctypes as C
import re
import subprocess

import pytest

import asd_b200 as asd
from conftest import ROOT

HEADER = ROOT / "include" / "asd_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n not in {"if", "while", "return", "sizeof"}))


def test_library_exports_every_declared_symbol():
    lib = asd.load()
    decl = declared_functions()
    assert set(decl) == set(asd.EXPORTED_SYMBOLS)
    out = subprocess.run(["nm", "-D", "--defined-only", str(asd.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    for name in decl:
        assert name in exported, name
        assert getattr(lib, name) is not None


def test_params_default_matches_reference_globals():
    p = asd.Params()
    assert asd.load().asd_params_default(C.byref(p), 100, 50) == asd.ASD_OK
    # llg_sqt_baseline.c:12-20, :172-173
    assert (p.N, p.nfile, p.J1, p.dt, p.vx, p.vy, p.spin_len) == (100, 50, 1.0, 0.02, 10, 10, 1.0)
    assert (p.J2, p.alpha, p.hx, p.hy, p.hz) == (0.0, 0.0, 0.0, 0.0, 0.0)


@pytest.mark.parametrize("kw", [dict(N=2, nfile=4), dict(N=8, nfile=0), dict(N=8, nfile=2, spin_len=0.0),
                                dict(N=8, nfile=2, dt=float("nan")), dict(N=8, nfile=2, J1=float("inf"))])
def test_create_rejects_bad_parameters(kw):
    N, nf = kw.pop("N"), kw.pop("nfile")
    p = asd.Params.make(N, nf, **kw)
    h = C.c_void_p()
    rc = asd.load().asd_ctx_create(C.byref(p), 0, C.byref(h))
    assert rc == asd.ASD_ERR_INVALID
    assert asd.last_error()
    assert not h.value


def test_null_arguments_are_errors():
    lib = asd.load()
    assert lib.asd_ctx_create(None, 0, None) == asd.ASD_ERR_INVALID
    assert lib.asd_ctx_step(None, 1) == asd.ASD_ERR_INVALID
    assert lib.asd_ctx_sqt(None, 0, None) == asd.ASD_ERR_INVALID
    assert lib.asd_set_params(0, 1, 1.0, 0.1) == asd.ASD_ERR_INVALID
    assert lib.asd_ctx_debug_poison(None) == asd.ASD_ERR_INVALID
    assert lib.asd_debug_fail_alloc(-1) == asd.ASD_ERR_INVALID
    assert lib.asd_debug_fail_alloc(0) == asd.ASD_OK


def test_no_cpu_fallback_without_gpu():
    """Without a device every computing call fails loudly; nothing runs on the CPU."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = asd.Params.make(8, 2)
    h = C.c_void_p()
    assert asd.load().asd_ctx_create(C.byref(p), 0, C.byref(h)) == asd.ASD_ERR_CUDA
