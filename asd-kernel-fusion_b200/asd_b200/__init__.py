"""Python binding of libasd_b200.so (ctypes).

This is the host-side mirror of the reference's interface for the hot path:
the reference's own entry points (``euler``, ``runge_kutta``, ``fused_dgemm``
with their argument meaning) and the context API that runs whole steps on the
GPU.  Spin arrays are float64 numpy arrays in the reference layout
``[nfile][N*N][3]`` (llg_sqt_baseline.c:185, :202).

The library is the product: this module only marshals arguments.  If the
shared library is missing the import fails; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_ROOT = Path(__file__).resolve().parent.parent
LIB_PATH = Path(os.environ.get("ASD_B200_LIB", PKG_ROOT / "lib" / "libasd_b200.so"))

ASD_OK = 0
ASD_ERR_INVALID = -1
ASD_ERR_CUDA = -2
ASD_ERR_NOMEM = -3
ASD_ERR_TIMEOUT = -4
ASD_ERR_STATE = -5
ASD_ERR_UNSUPPORTED = -6

LLG_STAGES = 0
LLG_FUSED_STEP = 1
LLG_AUTO = 2

SQT_FP64 = 0
SQT_TF32X3 = 1
SQT_BF16X3 = 2
SQT_FP16X3 = 3
MODE_NAMES = {SQT_FP64: "fp64", SQT_TF32X3: "tf32x3", SQT_BF16X3: "bf16x3",
              SQT_FP16X3: "fp16x3"}
MODES = {v: k for k, v in MODE_NAMES.items()}

# every symbol include/asd_b200.h declares
EXPORTED_SYMBOLS = (
    "asd_version", "asd_last_error", "asd_params_default", "asd_set_device",
    "asd_ctx_create", "asd_ctx_destroy", "asd_ctx_set_stream", "asd_ctx_get_params",
    "asd_ctx_set_params", "asd_ctx_loss_grad", "asd_ctx_loss_forward", "asd_ctx_loss_backward",
    "asd_ctx_set_spins", "asd_ctx_set_spins_device", "asd_ctx_get_spins",
    "asd_ctx_get_spins_device", "asd_ctx_step", "asd_ctx_sqt", "asd_ctx_sqt_async",
    "asd_ctx_sqt_magnitude",
    "asd_ctx_sqt_grid_async", "asd_ctx_sqt_grid",
    "asd_ctx_step_host", "asd_ctx_step_host_async", "asd_ctx_synchronize", "asd_ctx_set_ensemble", "asd_ctx_shard_origin_sums",
    "asd_ctx_shard_set_origin_sums", "asd_ctx_shard_sqt_async", "asd_ctx_shard_sqt_finish",
    "asd_ctx_set_llg_kernel", "asd_ctx_set_chunk_k",
    "asd_ctx_last_launches", "asd_ctx_time_kernels", "asd_ctx_kernel_time",
    "asd_ctx_check_device_status", "asd_debug_fail_alloc", "asd_ctx_debug_poison",
    "asd_check_bounded_wait", "asd_check_const_division", "asd_check_const_division_f32", "asd_umma_gemm_f32", "asd_sqt_split_noalloc",
    "asd_measure_fp64_peak", "asd_check_dmma_layout",
    "asd_spins_save", "asd_spins_load", "asd_batch_create", "asd_batch_destroy",
    "asd_batch_set_stream", "asd_batch_set_spins", "asd_batch_get_spins", "asd_batch_run",
    "asd_batch_configure", "asd_batch_configure_cluster", "asd_batch_autotune",
    "asd_batch_plan_clusters", "asd_set_params", "euler", "runge_kutta",
    "fused_dgemm", "asd_cblas_dgemm",
)


def _addr(x) -> int:
    """A device address: an int, or a tensor's data pointer."""
    return int(x.data_ptr()) if hasattr(x, "data_ptr") else int(x)


class AsdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"asd error {code}: {msg}")
        self.code = code


class Params(C.Structure):
    """asd_params (include/asd_b200.h)."""

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
        ("vx", C.c_int),
        ("vy", C.c_int),
    ]

    @classmethod
    def make(cls, N, nfile, J1=1.0, dt=0.02, J2=0.0, alpha=0.0, h=(0.0, 0.0, 0.0),
             spin_len=1.0, vx=None, vy=None):
        vx = N // 10 if vx is None else vx
        vy = N // 10 if vy is None else vy
        return cls(int(N), int(nfile), float(J1), float(J2), float(alpha), float(h[0]),
                   float(h[1]), float(h[2]), float(dt), float(spin_len), int(vx), int(vy))


_lib = None


def load() -> C.CDLL:
    """Loads libasd_b200.so once; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is not built; run __graft_entry__.build() or make -C "
                          f"{PKG_ROOT}")
    lib = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    dp = C.POINTER(C.c_double)
    P = C.POINTER(Params)
    sig = {
        "asd_version": ([], C.c_char_p),
        "asd_last_error": ([], C.c_char_p),
        "asd_params_default": ([P, C.c_int, C.c_int], C.c_int),
        "asd_set_device": ([C.c_int], C.c_int),
        "asd_ctx_create": ([P, C.c_uint, C.POINTER(vp)], C.c_int),
        "asd_ctx_destroy": ([vp], C.c_int),
        "asd_ctx_set_stream": ([vp, vp], C.c_int),
        "asd_ctx_get_params": ([vp, P], C.c_int),
        "asd_ctx_set_params": ([vp, P], C.c_int),
        "asd_ctx_loss_grad": ([vp, C.c_int, C.c_int, C.c_int, vp, dp, vp, vp], C.c_int),
        "asd_ctx_loss_forward": ([vp, C.c_int, C.c_int, C.c_int, vp, dp, vp], C.c_int),
        "asd_ctx_loss_backward": ([vp, vp, vp, vp], C.c_int),
        "asd_ctx_set_spins": ([vp, vp, C.c_int], C.c_int),
        "asd_ctx_set_spins_device": ([vp, vp, C.c_int], C.c_int),
        "asd_ctx_get_spins": ([vp, vp], C.c_int),
        "asd_ctx_get_spins_device": ([vp, vp], C.c_int),
        "asd_ctx_step": ([vp, C.c_int], C.c_int),
        "asd_ctx_sqt": ([vp, C.c_int, dp], C.c_int),
        "asd_ctx_sqt_async": ([vp, C.c_int, vp], C.c_int),
        "asd_ctx_sqt_magnitude": ([vp, dp], C.c_int),
        "asd_ctx_sqt_grid_async": ([vp, C.c_int, vp], C.c_int),
        "asd_ctx_sqt_grid": ([vp, C.c_int, vp], C.c_int),
        "asd_ctx_step_host": ([vp, vp, vp, C.c_int, dp], C.c_int),
        "asd_ctx_step_host_async": ([vp, vp, vp, C.c_int, vp], C.c_int),
        "asd_ctx_synchronize": ([vp], C.c_int),
        "asd_ctx_set_ensemble": ([vp, C.c_int], C.c_int),
        "asd_ctx_shard_origin_sums": ([vp, vp], C.c_int),
        "asd_ctx_shard_set_origin_sums": ([vp, vp], C.c_int),
        "asd_ctx_shard_sqt_async": ([vp, C.c_int, vp, vp], C.c_int),
        "asd_ctx_shard_sqt_finish": ([vp, vp, vp, vp], C.c_int),
        "asd_ctx_set_llg_kernel": ([vp, C.c_int], C.c_int),
        "asd_ctx_set_chunk_k": ([vp, C.c_int], C.c_int),
        "asd_ctx_last_launches": ([vp], C.c_int),
        "asd_ctx_time_kernels": ([vp, C.c_int], C.c_int),
        "asd_ctx_kernel_time": ([vp, C.c_int, dp, C.POINTER(C.c_int)], C.c_int),
        "asd_measure_fp64_peak": ([C.c_int, dp, dp, vp], C.c_int),
        "asd_check_dmma_layout": ([vp, vp, vp, vp], C.c_int),
        "asd_ctx_check_device_status": ([vp], C.c_int),
        "asd_debug_fail_alloc": ([C.c_long], C.c_int),
        "asd_ctx_debug_poison": ([vp], C.c_int),
        "asd_check_bounded_wait": ([C.c_int, C.c_uint, vp], C.c_int),
        "asd_check_const_division": ([vp, C.c_long, vp, vp], C.c_int),
        "asd_check_const_division_f32": ([vp, vp], C.c_int),
        "asd_umma_gemm_f32": ([C.c_int, C.c_long, C.c_int, vp, vp, vp, vp, vp, C.c_long, C.c_int,
                               vp],
                              C.c_int),
        "asd_sqt_split_noalloc": ([C.c_int, C.c_long, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp,
                                   C.c_double, C.c_double, C.c_int, vp, vp], C.c_int),
        "asd_batch_create": ([vp, C.c_int, C.POINTER(vp)], C.c_int),
        "asd_batch_destroy": ([vp], C.c_int),
        "asd_batch_set_stream": ([vp, vp], C.c_int),
        "asd_batch_set_spins": ([vp, C.c_int, vp], C.c_int),
        "asd_batch_get_spins": ([vp, C.c_int, vp], C.c_int),
        "asd_batch_run": ([vp, C.c_int], C.c_int),
        "asd_batch_configure": ([vp, C.c_int, C.c_int], C.c_int),
        "asd_batch_configure_cluster": ([vp, C.c_int, C.c_int], C.c_int),
        "asd_batch_plan_clusters": ([vp, C.c_int, C.c_int, C.c_int, C.c_long, vp, vp, C.c_int, vp,
                                     vp], C.c_int),
        "asd_batch_autotune": ([vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                C.POINTER(C.c_double)], C.c_int),
        "asd_spins_save": ([C.c_char_p, C.c_int, C.c_int, C.c_long, C.c_double, vp], C.c_int),
        "asd_spins_load": ([C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                            C.POINTER(C.c_long), C.POINTER(C.c_double), vp, C.c_size_t], C.c_int),
        "asd_set_params": ([C.c_int, C.c_int, C.c_double, C.c_double], C.c_int),
        "euler": ([vp, vp], None),
        "runge_kutta": ([vp] * 6, None),
        "fused_dgemm": ([C.POINTER(C.c_int)] * 3 + [dp, vp, C.POINTER(C.c_int), vp,
                                                   C.POINTER(C.c_int), vp, C.POINTER(C.c_int),
                                                   vp, vp], None),
        "asd_cblas_dgemm": ([C.c_int] * 6 + [C.c_double, vp, C.c_int, vp, C.c_int, C.c_double,
                                             vp, C.c_int], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def last_error() -> str:
    return load().asd_last_error().decode(errors="replace")


def _check(rc: int) -> None:
    if rc != ASD_OK:
        raise AsdError(rc, last_error())


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _as_spins(a, N, nfile) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.size != N * N * nfile * 3:
        raise ValueError(f"spins have {a.size} values, expected {nfile}x{N * N}x3")
    return a


def random_spins(N: int, nfile: int, seed: int, spin_len: float = 1.0) -> np.ndarray:
    """Seeded spins uniform on the sphere, [nfile][N*N][3] float64 (test and bench input;
    the reference's own initialisation is NaN, llg_sqt_baseline.c:196-206)."""
    rng = np.random.default_rng(seed)
    z = rng.uniform(-1.0, 1.0, size=(nfile, N * N))
    phi = rng.uniform(0.0, 2.0 * np.pi, size=(nfile, N * N))
    r = np.sqrt(1.0 - z * z)
    s = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=-1)
    return np.ascontiguousarray(s * spin_len, dtype=np.float64)


class Context:
    """asd_ctx: one lattice with nfile replicas resident on the GPU."""

    def __init__(self, params: Params, modes=None):
        lib = load()
        mask = 0
        for m in (modes or ()):
            mask |= 1 << (MODES[m] if isinstance(m, str) else int(m))
        h = C.c_void_p()
        _check(lib.asd_ctx_create(C.byref(params), mask, C.byref(h)))
        self._h = h
        self.params = params
        self.N = params.N
        self.nfile = params.nfile
        self._out = (C.c_double * 2)()

    def close(self) -> None:
        if self._h:
            load().asd_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def set_params(self, params: Params) -> None:
        _check(load().asd_ctx_set_params(self._h, C.byref(params)))
        self.params = params

    def loss_grad(self, nsteps: int, stride: int, checkpoint: int = 50, target=None):
        """asd_ctx_loss_grad: returns (loss, grad[6] = dL/d(J1, J2, alpha, hx, hy, hz),
        S(q,t_e) for e = 1..nsteps // stride as a complex array)."""
        E = nsteps // stride
        sq = np.zeros(2 * E)
        grad = np.zeros(6)
        loss = C.c_double(0.0)
        tgt = None
        if target is not None:
            t = np.asarray(target)
            tgt = np.ascontiguousarray(np.stack([t.real, t.imag], axis=-1).reshape(-1)
                                       if np.iscomplexobj(t) else t, dtype=np.float64)
            if tgt.size != 2 * E:
                raise ValueError(f"target has {tgt.size} values, expected {2 * E}")
        _check(load().asd_ctx_loss_grad(self._h, int(nsteps), int(stride), int(checkpoint),
                                        None if tgt is None else C.c_void_p(_ptr(tgt)),
                                        C.byref(loss), C.c_void_p(_ptr(grad)),
                                        C.c_void_p(_ptr(sq))))
        return loss.value, grad, sq[0::2] + 1j * sq[1::2]

    @staticmethod
    def _target(target, E):
        t = np.asarray(target)
        tgt = np.ascontiguousarray(np.stack([t.real, t.imag], axis=-1).reshape(-1)
                                   if np.iscomplexobj(t) else t, dtype=np.float64)
        if tgt.size != 2 * E:
            raise ValueError(f"target has {tgt.size} values, expected {2 * E}")
        return tgt

    def loss_forward(self, nsteps: int, stride: int, checkpoint: int = 50, target=None):
        """asd_ctx_loss_forward: (loss, S(q,t_e) as a complex array); keeps the
        tape for loss_backward."""
        E = nsteps // stride
        sq = np.zeros(2 * E)
        loss = C.c_double(0.0)
        tgt = None if target is None else self._target(target, E)
        _check(load().asd_ctx_loss_forward(self._h, int(nsteps), int(stride), int(checkpoint),
                                           None if tgt is None else C.c_void_p(_ptr(tgt)),
                                           C.byref(loss), C.c_void_p(_ptr(sq))))
        self._tape_E = E
        return loss.value, sq[0::2] + 1j * sq[1::2]

    def loss_backward(self, target):
        """asd_ctx_loss_backward: (grad[6] = dL/d(J1, J2, alpha, hx, hy, hz),
        dL/dtarget as a complex array d/dRe + i d/dIm)."""
        E = getattr(self, "_tape_E", 0)
        tgt = self._target(target, E)
        grad = np.zeros(6)
        dt = np.zeros(2 * E)
        _check(load().asd_ctx_loss_backward(self._h, C.c_void_p(_ptr(tgt)), C.c_void_p(_ptr(grad)),
                                            C.c_void_p(_ptr(dt))))
        return grad, dt[0::2] + 1j * dt[1::2]

    def set_stream(self, stream_ptr: int) -> None:
        _check(load().asd_ctx_set_stream(self._h, C.c_void_p(stream_ptr)))

    def set_spins(self, spins: np.ndarray, as_origin: bool = False) -> None:
        s = _as_spins(spins, self.N, self.nfile)
        _check(load().asd_ctx_set_spins(self._h, _ptr(s), int(as_origin)))

    def set_spins_device(self, dptr: int, as_origin: bool = False) -> None:
        _check(load().asd_ctx_set_spins_device(self._h, C.c_void_p(dptr), int(as_origin)))

    def get_spins(self) -> np.ndarray:
        out = np.empty((self.nfile, self.N * self.N, 3), dtype=np.float64)
        _check(load().asd_ctx_get_spins(self._h, _ptr(out)))
        return out

    def get_spins_device(self, dptr: int) -> None:
        _check(load().asd_ctx_get_spins_device(self._h, C.c_void_p(dptr)))

    def step(self, nsteps: int = 1) -> None:
        _check(load().asd_ctx_step(self._h, int(nsteps)))

    def sqt(self, mode=SQT_TF32X3) -> complex:
        mode = MODES[mode] if isinstance(mode, str) else int(mode)
        _check(load().asd_ctx_sqt(self._h, mode, self._out))
        return complex(self._out[0], self._out[1])

    def sqt_magnitude(self) -> float:
        """asd_ctx_sqt_magnitude: (1/M) sum_ij |C_ij - m_i . z_j| in FP64."""
        v = C.c_double(0.0)
        _check(load().asd_ctx_sqt_magnitude(self._h, C.byref(v)))
        return v.value

    def sqt_async(self, mode, d_out_ptr: int) -> None:
        mode = MODES[mode] if isinstance(mode, str) else int(mode)
        _check(load().asd_ctx_sqt_async(self._h, mode, C.c_void_p(d_out_ptr)))

    def sqt_grid_async(self, mode, d_out_ptr: int) -> None:
        mode = MODES[mode] if isinstance(mode, str) else int(mode)
        _check(load().asd_ctx_sqt_grid_async(self._h, mode, C.c_void_p(d_out_ptr)))

    def sqt_grid(self, mode=SQT_FP64) -> np.ndarray:
        """S(q,t) on the whole q grid as an N x N complex array [a, b] (q = 2 pi (a, b)/N)."""
        mode = MODES[mode] if isinstance(mode, str) else int(mode)
        v = np.empty(2 * self.N * self.N, dtype=np.float64)
        _check(load().asd_ctx_sqt_grid(self._h, mode, _ptr(v)))
        return (v[0::2] + 1j * v[1::2]).reshape(self.N, self.N)

    def step_host(self, spin_in_ptr: int, spin_out_ptr: int, mode=SQT_TF32X3) -> complex:
        mode = MODES[mode] if isinstance(mode, str) else int(mode)
        _check(load().asd_ctx_step_host(self._h, C.c_void_p(spin_in_ptr),
                                        C.c_void_p(spin_out_ptr), mode, self._out))
        return complex(self._out[0], self._out[1])

    def step_host_async(self, spin_in_ptr: int, spin_out_ptr: int, mode, sqt_out_ptr: int) -> None:
        """Enqueues one host-buffer step (pinned host or device pointers) and
        returns; the buffers are final after synchronize()."""
        mode = MODES[mode] if isinstance(mode, str) else int(mode)
        _check(load().asd_ctx_step_host_async(self._h, C.c_void_p(spin_in_ptr),
                                              C.c_void_p(spin_out_ptr), mode,
                                              C.c_void_p(sqt_out_ptr)))

    def synchronize(self) -> None:
        _check(load().asd_ctx_synchronize(self._h))

    # replica sharding of one ensemble (see asd_b200.shard) ------------------
    def set_ensemble(self, nfile_total: int) -> None:
        _check(load().asd_ctx_set_ensemble(self._h, int(nfile_total)))

    def shard_origin_sums(self, d_zsums) -> None:
        _check(load().asd_ctx_shard_origin_sums(self._h, C.c_void_p(_addr(d_zsums))))

    def shard_set_origin_sums(self, d_zsums) -> None:
        _check(load().asd_ctx_shard_set_origin_sums(self._h, C.c_void_p(_addr(d_zsums))))

    def shard_sqt_async(self, mode, d_part, d_sums) -> None:
        mode = MODES[mode] if isinstance(mode, str) else int(mode)
        _check(load().asd_ctx_shard_sqt_async(self._h, mode, C.c_void_p(_addr(d_part)),
                                              C.c_void_p(_addr(d_sums))))

    def shard_sqt_finish(self, d_part, d_sums, d_out) -> None:
        _check(load().asd_ctx_shard_sqt_finish(self._h, C.c_void_p(_addr(d_part)),
                                               C.c_void_p(_addr(d_sums)),
                                               C.c_void_p(_addr(d_out))))

    def set_llg_kernel(self, kernel) -> None:
        """"auto" (the default: the one-launch step where the lattice fills the
        GPU, else the stage kernels), "fused" (one launch per step) or
        "stages" (four launches, one per RK4 stage)."""
        k = {"fused": LLG_FUSED_STEP, "stages": LLG_STAGES, "auto": LLG_AUTO}.get(kernel, kernel)
        _check(load().asd_ctx_set_llg_kernel(self._h, int(k)))

    def set_chunk_k(self, chunk_k: int) -> None:
        _check(load().asd_ctx_set_chunk_k(self._h, int(chunk_k)))

    def last_launches(self) -> int:
        return int(load().asd_ctx_last_launches(self._h))

    def time_kernels(self, on: bool = True) -> None:
        """asd_ctx_time_kernels: record CUDA events around the RK4 step kernels
        and the S(q,t) GEMM on the stream each is launched on."""
        _check(load().asd_ctx_time_kernels(self._h, int(bool(on))))

    def kernel_time(self, which: str):
        """asd_ctx_kernel_time: (total ms, launches) of the timed RK4 step
        kernels ("llg") or S(q,t) GEMMs ("gemm") since the last read."""
        ms = C.c_double(0.0)
        n = C.c_int(0)
        _check(load().asd_ctx_kernel_time(self._h, {"llg": 0, "gemm": 1}[which], C.byref(ms),
                                          C.byref(n)))
        return ms.value, n.value

    def check_device_status(self) -> None:
        _check(load().asd_ctx_check_device_status(self._h))

    def debug_poison(self) -> None:
        """asd_ctx_debug_poison: NaN into every buffer that does not carry
        state between calls (tests of uninitialised reads)."""
        _check(load().asd_ctx_debug_poison(self._h))


def debug_fail_alloc(n: int) -> None:
    """asd_debug_fail_alloc: the n-th device allocation of the context API
    from now on fails with ASD_ERR_NOMEM (0 switches it off)."""
    _check(load().asd_debug_fail_alloc(int(n)))


# ------------------------------------------------------------ drop-in layer
def set_params(N: int, nfile: int, J1: float = 1.0, dt: float = 0.02) -> None:
    """asd_set_params: the globals the reference's functions read."""
    _check(load().asd_set_params(int(N), int(nfile), float(J1), float(dt)))


def euler(spin: np.ndarray) -> np.ndarray:
    """The reference's euler(spin0, derivative) (llg_sqt_baseline.c:29)."""
    s = np.ascontiguousarray(spin, dtype=np.float64)
    d = np.full_like(s, np.nan)
    load().euler(_ptr(s), _ptr(d))
    return d


def runge_kutta(spin: np.ndarray):
    """The reference's runge_kutta (llg_sqt_baseline.c:95); returns cur, k1..k4."""
    s = np.ascontiguousarray(spin, dtype=np.float64)
    outs = [np.full_like(s, np.nan) for _ in range(5)]
    load().runge_kutta(_ptr(s), *[_ptr(o) for o in outs])
    return tuple(outs)


def fused_dgemm(m, n, k, alpha, a, lda, b, ldb, c, ldc, q, sum_):
    """The reference's fused_dgemm (kernel_fusion/gemm_kernel.h:355); updates c and sum_
    in place."""
    ci = lambda v: C.byref(C.c_int(int(v)))
    al = C.c_double(float(alpha))
    for arr in (a, b, c, q, sum_):
        if not (arr.dtype == np.float64 and arr.flags.c_contiguous):
            raise ValueError("fused_dgemm arrays must be C-contiguous float64")
    load().fused_dgemm(ci(m), ci(n), ci(k), C.byref(al), _ptr(a), ci(lda), _ptr(b), ci(ldb),
                       _ptr(c), ci(ldc), _ptr(q), _ptr(sum_))


CBLAS_ROW_MAJOR, CBLAS_COL_MAJOR = 101, 102
CBLAS_NO_TRANS, CBLAS_TRANS, CBLAS_CONJ_TRANS = 111, 112, 113


def cblas_dgemm(order, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc) -> None:
    """asd_cblas_dgemm, the reference's cblas_dgemm (gemm/llg_sqt_mkl.c:378) on the GPU,
    on host float64 arrays (a and b may be None where BLAS reads neither); c is updated
    in place."""
    for arr in (a, b, c):
        if arr is not None and not (arr.dtype == np.float64 and arr.flags.c_contiguous):
            raise ValueError("cblas_dgemm arrays must be C-contiguous float64")
    ptr = lambda arr: None if arr is None else C.c_void_p(arr.ctypes.data)
    _check(load().asd_cblas_dgemm(int(order), int(transa), int(transb), int(m), int(n), int(k),
                                  float(alpha), ptr(a), int(lda), ptr(b), int(ldb), float(beta),
                                  ptr(c), int(ldc)))


def umma_gemm_f32(kind: int, rows: int, Kp: int, a_hi: int, a_lo: int, b_hi: int, b_lo: int,
                  c: int, ldc: int, chunk_k: int = 0, stream: int = 0) -> None:
    """asd_umma_gemm_f32 on device pointers (diagnostic)."""
    _check(load().asd_umma_gemm_f32(int(kind), int(rows), int(Kp), C.c_void_p(a_hi),
                                    C.c_void_p(a_lo), C.c_void_p(b_hi), C.c_void_p(b_lo),
                                    C.c_void_p(c), int(ldc), int(chunk_k), C.c_void_p(stream)))


def measure_fp64_peak(which: str, stream: int = 0):
    """asd_measure_fp64_peak: (TFLOP/s, ms) of the FP64 FMA ("fma") or FP64
    tensor-core MMA ("dmma") throughput kernel on the current device."""
    tf = C.c_double(0.0)
    ms = C.c_double(0.0)
    _check(load().asd_measure_fp64_peak({"fma": 0, "dmma": 1}[which], C.byref(tf), C.byref(ms),
                                        C.c_void_p(stream)))
    return tf.value, ms.value


def check_dmma_layout(A: int, B: int, D: int, stream: int = 0) -> None:
    """asd_check_dmma_layout on device pointers (diagnostic)."""
    _check(load().asd_check_dmma_layout(C.c_void_p(A), C.c_void_p(B), C.c_void_p(D),
                                        C.c_void_p(stream)))


def sqt_split_noalloc(kind: int, rows: int, Kp: int, a_hi: int, a_lo: int, b_hi: int, b_lo: int,
                      row4: int, row1: int, col4: int, col1: int, alpha: float, scale: float,
                      chunk_k: int, d_out: int, stream: int = 0) -> None:
    """asd_sqt_split_noalloc on device pointers: S(q,t) without any allocation."""
    v = C.c_void_p
    _check(load().asd_sqt_split_noalloc(int(kind), int(rows), int(Kp), v(a_hi), v(a_lo), v(b_hi),
                                        v(b_lo), v(row4), v(row1), v(col4), v(col1),
                                        float(alpha), float(scale), int(chunk_k), v(d_out),
                                        v(stream)))


def check_const_division(x_ptr: int, n: int, bad_ptr: int, stream: int = 0) -> None:
    """asd_check_const_division on device pointers (diagnostic)."""
    _check(load().asd_check_const_division(C.c_void_p(x_ptr), int(n), C.c_void_p(bad_ptr),
                                           C.c_void_p(stream)))


def check_const_division_f32(bad_ptr: int, stream: int = 0) -> None:
    """asd_check_const_division_f32: all 2^32 float patterns (diagnostic)."""
    _check(load().asd_check_const_division_f32(C.c_void_p(bad_ptr), C.c_void_p(stream)))


def save_spins(path, spins: np.ndarray, step: int = 0, spin_len: float = 1.0) -> None:
    """asd_spins_save: spins [nfile][N*N][3] float64 to a checkpoint file."""
    s = np.ascontiguousarray(spins, dtype=np.float64)
    nfile, M, _ = s.shape
    N = int(round(M ** 0.5))
    _check(load().asd_spins_save(str(path).encode(), N, nfile, int(step), float(spin_len),
                                 _ptr(s)))


def load_spins(path):
    """asd_spins_load: returns (spins [nfile][N*N][3], step, spin_len)."""
    N, nf, st, sl = C.c_int(), C.c_int(), C.c_long(), C.c_double()
    lib = load()
    _check(lib.asd_spins_load(str(path).encode(), C.byref(N), C.byref(nf), C.byref(st),
                              C.byref(sl), None, 0))
    out = np.empty((nf.value, N.value * N.value, 3), dtype=np.float64)
    _check(lib.asd_spins_load(str(path).encode(), C.byref(N), C.byref(nf), C.byref(st),
                              C.byref(sl), C.c_void_p(_ptr(out)), out.size))
    return out, st.value, sl.value


class Lattice(C.Structure):
    """asd_lattice: one lattice of a batch."""

    _fields_ = [("N", C.c_int), ("J1", C.c_double), ("J2", C.c_double), ("alpha", C.c_double),
                ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double), ("dt", C.c_double),
                ("spin_len", C.c_double)]

    @classmethod
    def make(cls, N, J1=1.0, J2=0.0, alpha=0.0, h=(0.0, 0.0, 0.0), dt=0.01, spin_len=1.0):
        return cls(int(N), float(J1), float(J2), float(alpha), float(h[0]), float(h[1]),
                   float(h[2]), float(dt), float(spin_len))


class Batch:
    """asd_batch: independent lattices stepped by one persistent launch."""

    def __init__(self, lattices):
        self.lattices = list(lattices)
        arr = (Lattice * len(self.lattices))(*self.lattices)
        h = C.c_void_p()
        _check(load().asd_batch_create(arr, len(self.lattices), C.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            load().asd_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_spins(self, l: int, spins: np.ndarray) -> None:
        s = np.ascontiguousarray(spins, dtype=np.float32)
        if s.size != self.lattices[l].N ** 2 * 3:
            raise ValueError("spins must be float32 [N*N][3]")
        _check(load().asd_batch_set_spins(self._h, int(l), C.c_void_p(_ptr(s))))

    def get_spins(self, l: int) -> np.ndarray:
        N = self.lattices[l].N
        out = np.empty((N * N, 3), dtype=np.float32)
        _check(load().asd_batch_get_spins(self._h, int(l), C.c_void_p(_ptr(out))))
        return out

    def run(self, nsteps: int) -> None:
        _check(load().asd_batch_run(self._h, int(nsteps)))

    def configure(self, tile: int, ctas_per_sm: int) -> None:
        """Global-memory kernel with this work decomposition."""
        _check(load().asd_batch_configure(self._h, int(tile), int(ctas_per_sm)))

    def configure_cluster(self, cluster_size: int, threads: int = 0) -> None:
        """Cluster-resident kernel (raises AsdError if the batch does not fit)."""
        _check(load().asd_batch_configure_cluster(self._h, int(cluster_size), int(threads)))

    def autotune(self, trial_steps: int = 20):
        t, c, ms = C.c_int(), C.c_int(), C.c_double()
        _check(load().asd_batch_autotune(self._h, int(trial_steps), C.byref(t), C.byref(c),
                                         C.byref(ms)))
        return t.value, c.value, ms.value


def batch_plan_clusters(sizes, cluster_size: int, clusters: int, smem_limit: int = 232448):
    """asd_batch_plan_clusters (host only): (ctas [n][4], segs [m][12], smem
    bytes, fits) -- see the header for the columns."""
    sz = np.ascontiguousarray(sizes, dtype=np.int32)
    ctas = np.zeros((clusters * cluster_size, 4), dtype=np.int32)
    cap = int(sum(int(n) for n in sizes) + clusters * cluster_size)
    segs = np.zeros((cap, 12), dtype=np.int32)
    nsegs, smem = C.c_int(), C.c_long()
    rc = load().asd_batch_plan_clusters(_ptr(sz), len(sz), int(cluster_size), int(clusters),
                                        int(smem_limit), _ptr(ctas), _ptr(segs), cap,
                                        C.byref(nsegs), C.byref(smem))
    if rc not in (ASD_OK, ASD_ERR_UNSUPPORTED):
        _check(rc)
    return ctas, segs[: nsegs.value], smem.value, rc == ASD_OK


def noisy_ordered_spins(N: int, eta: float, seed: int) -> np.ndarray:
    """An ordered state along z with Gaussian noise of amplitude eta, renormalised
    (the "temperature" of a lattice in an ensemble), float64 [N*N][3]."""
    rng = np.random.default_rng(seed)
    s = np.zeros((N * N, 3))
    s[:, 2] = 1.0
    s += eta * rng.standard_normal((N * N, 3))
    return s / np.linalg.norm(s, axis=-1, keepdims=True)
