"""ctypes loaders for the CPU oracle.

TEST INFRASTRUCTURE ONLY: tests/, ``__graft_entry__.smoke()`` and the CPU arms
of ``bench.py`` use this module as the checker or as the timed CPU baseline.
The product path (the CUDA library) never imports it.

* ``Oracle``   -- oracle/liboracle.so, the C restatement (asd_oracle.c).
* ``RefLib``   -- oracle/_ref/libref_<variant>.so, the reference's own programs
  compiled from their sources by ``make -C oracle ref`` plus the harness in
  ref_glue.c.  Present only where the build ran (this container, or a GPU box
  that received the prebuilt files).

Spin arrays are float64 numpy arrays in the reference layout
``[nfile][N*N][3]`` (llg_sqt_baseline.c:185, :202), C-contiguous.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class OracleParams(C.Structure):
    _fields_ = [
        ("N", C.c_int),
        ("nfile", C.c_int),
        ("J1", C.c_double),
        ("J2", C.c_double),
        ("alpha", C.c_double),
        ("hx", C.c_double),
        ("hy", C.c_double),
        ("hz", C.c_double),
        ("dt", C.c_double),
        ("spin_len", C.c_double),
    ]


def build(quiet: bool = True) -> None:
    """Compile liboracle.so, and the reference libraries when the sources exist."""
    kw = dict(cwd=HERE, check=True)
    if quiet:
        kw.update(stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    subprocess.run(["make", "liboracle.so"], **kw)
    ref = Path(os.environ.get("ASD_REFERENCE", "")).expanduser()
    if os.environ.get("ASD_REFERENCE") and (ref / "baseline" / "llg_sqt_baseline.c").exists():
        subprocess.run(["make", "ref", f"REF={ref}"], **kw)


def make_params(N, nfile, J1=1.0, dt=0.02, J2=0.0, alpha=0.0, h=(0.0, 0.0, 0.0), spin_len=1.0):
    return OracleParams(int(N), int(nfile), float(J1), float(J2), float(alpha),
                        float(h[0]), float(h[1]), float(h[2]), float(dt), float(spin_len))


class Oracle:
    """The C restatement of the reference's hot path."""

    def __init__(self, path: Path | None = None):
        path = Path(path) if path else HERE / "liboracle.so"
        if not path.exists():
            build()
        lib = C.CDLL(str(path))
        P = C.POINTER(OracleParams)
        lib.oracle_llg_deriv.argtypes = [P, _dp, _dp]
        lib.oracle_rk4.argtypes = [P, _dp, _dp, _dp, _dp, _dp, _dp]
        lib.oracle_renorm.argtypes = [P, _dp, _dp]
        lib.oracle_steps.argtypes = [P, _dp, C.c_int]
        lib.oracle_steps.restype = C.c_int
        for name in ("oracle_sqt_gemm", "oracle_sqt_direct", "oracle_sqt_fused", "oracle_sqt_factorized"):
            getattr(lib, name).argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp]
        fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
        lib.oracle_steps_f32.argtypes = [P, fp, C.c_int]
        lib.oracle_steps_f32.restype = C.c_int
        lib.oracle_sqt_grid.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp]
        lib.oracle_fused_dgemm.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, _dp, C.c_int,
                                           _dp, C.c_int, _dp, C.c_int, _dp, _dp]
        self.lib = lib

    # LLG -----------------------------------------------------------------
    def deriv(self, p: OracleParams, spin: np.ndarray) -> np.ndarray:
        out = np.empty_like(spin)
        self.lib.oracle_llg_deriv(C.byref(p), np.ascontiguousarray(spin), out)
        return out

    def rk4(self, p: OracleParams, spin: np.ndarray):
        spin = np.ascontiguousarray(spin)
        cur, k1, k2, k3, k4 = (np.empty_like(spin) for _ in range(5))
        self.lib.oracle_rk4(C.byref(p), spin, cur, k1, k2, k3, k4)
        return cur, k1, k2, k3, k4

    def renorm(self, p: OracleParams, cur: np.ndarray) -> np.ndarray:
        out = np.empty_like(cur)
        self.lib.oracle_renorm(C.byref(p), np.ascontiguousarray(cur), out)
        return out

    def steps(self, p: OracleParams, spin: np.ndarray, nsteps: int) -> np.ndarray:
        s = np.array(spin, dtype=np.float64, copy=True, order="C")
        if self.lib.oracle_steps(C.byref(p), s, int(nsteps)) != 0:
            raise MemoryError("oracle_steps")
        return s

    def steps_f32(self, p: OracleParams, spin: np.ndarray, nsteps: int) -> np.ndarray:
        """FP32 RK4 + FP64 renormalisation, one replica, float32 [N*N][3]."""
        s = np.array(spin, dtype=np.float32, copy=True, order="C")
        if self.lib.oracle_steps_f32(C.byref(p), s, int(nsteps)) != 0:
            raise MemoryError("oracle_steps_f32")
        return s

    # S(q,t) --------------------------------------------------------------
    def _sqt(self, fn, N, nfile, vx, vy, spin_t, spin_0) -> complex:
        out = np.zeros(2)
        fn(int(N), int(nfile), int(vx), int(vy), np.ascontiguousarray(spin_t),
           np.ascontiguousarray(spin_0), out)
        return complex(out[0], out[1])

    def sqt_gemm(self, N, nfile, vx, vy, spin_t, spin_0) -> complex:
        return self._sqt(self.lib.oracle_sqt_gemm, N, nfile, vx, vy, spin_t, spin_0)

    def sqt_direct(self, N, nfile, vx, vy, spin_t, spin_0) -> complex:
        return self._sqt(self.lib.oracle_sqt_direct, N, nfile, vx, vy, spin_t, spin_0)

    def sqt_fused(self, N, nfile, vx, vy, spin_t, spin_0) -> complex:
        return self._sqt(self.lib.oracle_sqt_fused, N, nfile, vx, vy, spin_t, spin_0)

    def sqt_factorized(self, N, nfile, vx, vy, spin_t, spin_0) -> complex:
        return self._sqt(self.lib.oracle_sqt_factorized, N, nfile, vx, vy, spin_t, spin_0)

    def sqt_grid(self, N, nfile, spin_t, spin_0) -> np.ndarray:
        re = np.zeros(N * N)
        im = np.zeros(N * N)
        self.lib.oracle_sqt_grid(int(N), int(nfile), np.ascontiguousarray(spin_t),
                                 np.ascontiguousarray(spin_0), re, im)
        return (re + 1j * im).reshape(N, N)

    def fused_dgemm(self, m, n, k, alpha, a, lda, b, ldb, c, ldc, q, sum_):
        self.lib.oracle_fused_dgemm(m, n, k, alpha, a, lda, b, ldb, c, ldc, q, sum_)


class RefLib:
    """The reference's own compiled program for one variant (baseline, fusion, gemm)."""

    def __init__(self, variant: str):
        path = REF_DIR / f"libref_{variant}.so"
        if not path.exists():
            raise FileNotFoundError(path)
        lib = C.CDLL(str(path))
        lib.ref_setup.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int]
        lib.ref_setup.restype = C.c_int
        lib.ref_get_vx.restype = C.c_int
        lib.ref_euler.argtypes = [_dp, _dp]
        lib.ref_runge_kutta.argtypes = [_dp] * 6
        lib.ref_steps.argtypes = [_dp, C.c_int, C.c_double]
        lib.ref_steps.restype = C.c_int
        lib.ref_steps_timed.argtypes = [_dp, C.c_int, C.c_double, C.POINTER(C.c_double)]
        lib.ref_steps_timed.restype = C.c_int
        if variant == "fusion":
            lib.ref_fusion_init.argtypes = [_dp, C.c_long]
            lib.ref_fusion_init.restype = C.c_int
            lib.ref_fusion_sqt.argtypes = [_dp, _dp]
            lib.ref_fusion_sqt.restype = C.c_int
            lib.ref_fusion_sqt_timed.argtypes = [_dp, _dp, C.POINTER(C.c_double),
                                                 C.POINTER(C.c_double)]
            lib.ref_fusion_sqt_timed.restype = C.c_int
            lib.ref_fused_dgemm.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, _dp, C.c_int,
                                            _dp, C.c_int, _dp, C.c_int, _dp, _dp]
        if variant == "gemm":
            lib.ref_gemm_sqt.argtypes = [_dp, _dp, _dp]
            lib.ref_gemm_sqt.restype = C.c_int
            lib.ref_gemm_sqt_band.argtypes = [_dp, _dp, C.c_long, _dp, C.POINTER(C.c_double),
                                              C.POINTER(C.c_double)]
            lib.ref_gemm_sqt_band.restype = C.c_int
        self.lib = lib
        self.variant = variant
        self.threads = 1

    @staticmethod
    def available(variant: str) -> bool:
        return (REF_DIR / f"libref_{variant}.so").exists()

    def setup(self, N, nfile, J1=1.0, dt=0.02, threads=0) -> int:
        self.threads = self.lib.ref_setup(int(N), int(nfile), float(J1), float(dt), int(threads))
        return self.threads

    def euler(self, spin):
        out = np.empty_like(spin)
        self.lib.ref_euler(np.ascontiguousarray(spin), out)
        return out

    def runge_kutta(self, spin):
        spin = np.array(spin, dtype=np.float64, copy=True, order="C")
        cur, k1, k2, k3, k4 = (np.empty_like(spin) for _ in range(5))
        self.lib.ref_runge_kutta(spin, cur, k1, k2, k3, k4)
        return cur, k1, k2, k3, k4

    def steps(self, spin, nsteps, spin_len=1.0):
        s = np.array(spin, dtype=np.float64, copy=True, order="C")
        if self.lib.ref_steps(s, int(nsteps), float(spin_len)) != 0:
            raise MemoryError("ref_steps")
        return s

    def step_time(self, spin, spin_len=1.0) -> float:
        """Seconds of one runge_kutta + renormalisation step of the reference
        on `spin` (a second step, timed after a first that touches the work
        buffers, as main's loop reuses them)."""
        s = np.array(spin, dtype=np.float64, copy=True, order="C")
        t = C.c_double(0.0)
        if self.lib.ref_steps_timed(s, 2, float(spin_len), C.byref(t)) != 0:
            raise MemoryError("ref_steps_timed")
        return t.value

    def fusion_sqt_timed(self, spin_t):
        """(S(q,t) over the band, seconds of the O(M K) pack, seconds of the band)."""
        out = np.zeros(2)
        tp, tb = C.c_double(0.0), C.c_double(0.0)
        if self.lib.ref_fusion_sqt_timed(np.ascontiguousarray(spin_t), out, C.byref(tp),
                                         C.byref(tb)) != 0:
            raise RuntimeError("ref_fusion_sqt_timed")
        return complex(out[0], out[1]), tp.value, tb.value

    def gemm_sqt_band(self, spin_t, spin_0, rows):
        """The gemm program's S(q,t) over the first `rows` rows of C:
        (value over the band, seconds of the O(M K) packs, seconds of the band)."""
        out = np.zeros(2)
        tp, tb = C.c_double(0.0), C.c_double(0.0)
        if self.lib.ref_gemm_sqt_band(np.ascontiguousarray(spin_t), np.ascontiguousarray(spin_0),
                                      int(rows), out, C.byref(tp), C.byref(tb)) != 0:
            raise MemoryError("ref_gemm_sqt_band")
        return complex(out[0], out[1]), tp.value, tb.value

    def fusion_init(self, spin_0, rows=0):
        rc = self.lib.ref_fusion_init(np.ascontiguousarray(spin_0), int(rows))
        if rc != 0:
            raise MemoryError(f"ref_fusion_init rc={rc}")

    def fusion_sqt(self, spin_t) -> complex:
        out = np.zeros(2)
        self.lib.ref_fusion_sqt(np.ascontiguousarray(spin_t), out)
        return complex(out[0], out[1])

    def gemm_sqt(self, spin_t, spin_0) -> complex:
        out = np.zeros(2)
        if self.lib.ref_gemm_sqt(np.ascontiguousarray(spin_t), np.ascontiguousarray(spin_0), out) != 0:
            raise MemoryError("ref_gemm_sqt")
        return complex(out[0], out[1])


def random_spins(N: int, nfile: int, seed: int, spin_len: float = 1.0) -> np.ndarray:
    """Seeded spins uniform on the sphere, [nfile][N*N][3] float64."""
    rng = np.random.default_rng(seed)
    z = rng.uniform(-1.0, 1.0, size=(nfile, N * N))
    phi = rng.uniform(0.0, 2.0 * np.pi, size=(nfile, N * N))
    r = np.sqrt(1.0 - z * z)
    s = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=-1)
    return np.ascontiguousarray(s * spin_len, dtype=np.float64)
