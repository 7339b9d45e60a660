#!/usr/bin/env python
"""Benchmark of the hot path: per step, one RK4 step of the LLG equation for
every replica and one S(q,t) evaluation (the correlation GEMM with its fused
phase epilogue).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload sqt256|sqt128|grid32|adjoint64|batch48]

Default workload: the 256 x 256 lattice with 1000 replicas (J = 1,
J2 = -0.3, alpha = 0.02, h = 0, dt = 0.005), S(q,t) in BF16x3 split precision
-- a GEMM of M = 65536 sites by K = 3000 per step.  ``sqt128`` is the
128 x 128 lattice with 500 replicas (J = -1, h = (0, 0, 0.5), alpha = 0.05,
dt = 0.005), S(q,t) in TF32x3.

Prints one JSON line on rank 0.  ``value`` is the whole job's throughput in
site-steps/s (a site-step = one spin of one replica advanced one RK4 step,
with the step's S(q,t) evaluation included), spins resident in HBM.  ``e2e``
is the same metric through asd_ctx_step_host_async: the spins come from
pinned host memory and go back every step, as the reference's runge_kutta
contract has them.  The roofline is that of the S(q,t) GEMM, the dominant
kernel, whose duration is measured by CUDA events on its own stream inside
the timed region.  Under torchrun every rank runs its own lattice (weak
scaling, no collective in the data path); the time is the max over ranks.

``--impl reference`` times the reference's own C programs (oracle/_ref,
compiled from its sources) on the host cores for the same workload, each step
a bounded sample: runge_kutta + renormalisation on a subset of the replicas
and the S(q,t) of its fused-AVX2 and OpenBLAS programs on a band of GEMM rows,
each scaled to the whole workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "asd-kernel-fusion_b200"))

METRIC = "LLG site-steps/s + S(q,t) GEMM TFLOP/s, mixed vs FP64 plain at stated error"
WORKLOADS = {
    "sqt256": dict(N=256, nfile=1000, J1=1.0, J2=-0.3, alpha=0.02, h=(0.0, 0.0, 0.0), dt=0.005,
                   mode="bf16x3",
                   desc="llg-rk4+sqt 256x256 lattice, 1000 replicas, J=1, J2=-0.3, alpha=0.02, "
                        "dt=0.005, S(q,t) in BF16x3"),
    "sqt128": dict(N=128, nfile=500, J1=-1.0, J2=0.0, alpha=0.05, h=(0.0, 0.0, 0.5), dt=0.005,
                   mode="tf32x3",
                   desc="llg-rk4+sqt 128x128 lattice, 500 replicas, J=-1, h=(0,0,0.5), "
                        "alpha=0.05, dt=0.005, S(q,t) in TF32x3"),
}
LLG_BYTES_PER_SITE_STEP = 384  # 4 fused stage kernels: 3+5+5+3 FP64 3-vectors
LLG_FUSED_BYTES_PER_SITE_STEP = 48  # one streamed step: read y, write y
DEFAULT_CHUNK_K = {"tf32x3": 512, "bf16x3": 1024, "fp16x3": 1024}


def llg_fp64_ops(J2: bool, H: bool, damp: bool) -> int:
    """FP64 operations of one site-step as the kernels write them (add, sub,
    mul and fma 1 each; a division or square root 1 each, although the
    hardware runs a short sequence for them): the right-hand side (exchange
    12 mul + 12 add, J2 as much again, the field 3 add, H x S 9, damping 18)
    and dt * f (3) in each of the 4 stages, then the stage combinations
    (18 + 18 + 15) and stage 4's combination and renormalisation (24)."""
    rhs = 24 + (24 if J2 else 0) + (3 if H else 0) + 9 + (18 if damp else 0)
    return 4 * (rhs + 3) + 18 + 18 + 15 + 24


def measured_peaks():
    """HBM GB/s and dense BF16 TFLOP/s of this pool's B200s (MEASURED_PEAKS.json,
    written per machine), else the earlier measurement on this pool."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "bf16_burst": d.get("bf16_tflops", 1590.0),
                "bf16_sustained": d.get("bf16_tflops_sustained", d.get("bf16_tflops", 1400.0)),
                "source": "measured (MEASURED_PEAKS.json)"}
    return {"hbm_gbs": 6650.0, "bf16_burst": 1590.0, "bf16_sustained": 1400.0,
            "source": "fallback (earlier measurement on this pool)"}


def split_ceiling(mode, frac):
    """The highest useful-flop fraction of the dense BF16 peak a 3-term split
    GEMM can reach: three tensor-core products per useful one, FP16 products
    run at the BF16 rate and TF32 ones at half of it on B200.  frac_of_ceiling is how close
    the kernel is to that bound."""
    ceil = {"tf32x3": 1.0 / 6.0, "bf16x3": 1.0 / 3.0, "fp16x3": 1.0 / 3.0}.get(mode)
    if ceil is None or frac is None:
        return {}
    return {"split_ceiling_frac": ceil, "frac_of_split_ceiling": frac / ceil}


def sustained_fma_peak(asd, stream, device, seconds=0.3):
    """The FP64 FMA issue rate held for `seconds` back to back (the one-launch
    LLG step runs long enough for the power cap to lower the SM clock, as a
    ~1 ms burst does not): median TFLOP/s of the repeated peak kernel and the
    SM clock sampled meanwhile."""
    tfs = []
    with ClockSampler(device) as clk:
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < seconds:
            tfs.append(asd.measure_fp64_peak("fma", stream.cuda_stream)[0])
    return statistics.median(tfs), clk.summary()


def add_per_clock(llg, llg_clocks, fma_clocks):
    """Per LLG kernel, the FP64 fraction at equal SM clocks: the fraction of
    the sustained FMA rate times (FMA clock / the kernel's clock), where both
    median clocks were sampled (ops per cycle against FMAs per cycle)."""
    fmhz = (fma_clocks or {}).get("sm_mhz")
    for k, e in llg.items():
        kmhz = ((llg_clocks or {}).get(k) or {}).get("sm_mhz")
        if fmhz and kmhz and e.get("fp64_frac_sustained") is not None:
            e["sm_mhz"] = kmhz
            e["fp64_frac_per_clock"] = e["fp64_frac_sustained"] * fmhz / kmhz
    return llg


def llg_report(ms_by_kernel, sites_replicas, ops, hbm, fma_tops, fma_sustained_tops=None):
    """Per LLG kernel: site-steps/s, DRAM bytes against the HBM peak (the
    bound of the stage kernels) and FP64 operations against the measured FP64
    FMA issue rate (the bound of the one-launch step): the burst figure and,
    where given, the rate the same GPU holds under its power cap."""
    out = {}
    for k, ms in ms_by_kernel.items():
        bps = LLG_BYTES_PER_SITE_STEP if k == "stages" else LLG_FUSED_BYTES_PER_SITE_STEP
        rate = sites_replicas / (ms / 1e3)
        out[k] = {"site_steps_per_s": rate, "ms": ms, "bytes_per_site_step": bps,
                  "achieved_gbs": bps * rate / 1e9, "hbm_peak_gbs": hbm,
                  "frac": bps * rate / 1e9 / hbm, "fp64_ops_per_site_step": ops,
                  "achieved_fp64_tops": ops * rate / 1e12,
                  "fp64_fma_peak_tops": fma_tops,
                  "fp64_frac": ops * rate / 1e12 / fma_tops if fma_tops else None,
                  "bound": "hbm" if k == "stages" else "fp64"}
        if fma_sustained_tops:
            out[k]["fp64_fma_sustained_tops"] = fma_sustained_tops
            out[k]["fp64_frac_sustained"] = ops * rate / 1e12 / fma_sustained_tops
    return out


def aggregate(ms_per_step: float, units_per_rank: float, world: int, dist=None, device=None):
    """Whole-job throughput of a weak-scaling run: every rank processed
    units_per_rank units in ms_per_step on its own clock; the job's time is
    the slowest rank's.  Returns (max ms over ranks, units per second)."""
    if world > 1 and dist is not None:
        import torch

        t = torch.tensor([ms_per_step], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_per_step = float(t.item())
    return ms_per_step, world * units_per_rank / (ms_per_step / 1e3)


def rank_seed(rank: int) -> int:
    """Each rank steps its own lattice (independent ensembles)."""
    return rank


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def bench_config(name: str, args) -> dict:
    """The workload description both arms print, key for key."""
    w = WORKLOADS[name]
    N, nf = w["N"], w["nfile"]
    M, K = N * N, 3 * nf
    mode = args.mode or w["mode"]
    state_mb = M * K * 8 / 1e6
    label = {"fp64": "FP64", "tf32x3": "TF32x3", "bf16x3": "BF16x3", "fp16x3": "FP16x3"}
    desc = w["desc"].replace(f"S(q,t) in {label[w['mode']]}", f"S(q,t) in {label[mode]}")
    return {"workload": desc, "sites": M, "replicas": nf, "gemm_m": M, "gemm_n": M,
            "gemm_k": K, "sqt_mode": mode, "llg_kernel": args.llg_kernel,
            "chunk_k": args.chunk_k if args.chunk_k >= 0 else DEFAULT_CHUNK_K.get(mode, 0),
            "l2": f"inputs larger than L2 (spin state {state_mb:.0f} MB per array)"}


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    REASONS = {
        "gpu_idle": 0x1, "applications_clocks_setting": 0x2, "sw_power_cap": 0x4,
        "hw_slowdown": 0x8, "sync_boost": 0x10, "sw_thermal_slowdown": 0x20,
        "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80,
    }

    def __init__(self, device_index: int, period: float = 0.005):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self.period = period
        self._stop = threading.Event()
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                bits = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for name, b in self.REASONS.items():
                    if bits & b:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self.nv:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *exc):
        if self.nv:
            self._stop.set()
            self.t.join()

    def summary(self):
        med = statistics.median(self.samples) if self.samples else None
        return {"sm_mhz": med, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


# --------------------------------------------------------------- CPU arms
def _orc():
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc

    return orc


class CpuReference:
    """The reference's own compiled programs (oracle/_ref, built from its
    sources) on the host cores, for one workload, in bounded samples:

    * LLG: runge_kutta + renormalisation (llg_sqt_baseline.c:95-142, :298-309)
      on the first `llg_replicas` replicas, scaled to all of them (replicas
      are independent, the cost is linear in them);
    * S(q,t), fused-AVX2 program (llg_sqt_fusion.c:370-441 around
      fused_dgemm) and OpenBLAS program (gemm/llg_sqt_mkl.c:369-423 around
      cblas_dgemm): the per-step A pack and replica means (O(M K), timed
      whole) plus the GEMM and its epilogue on a band of C's rows (O(rows M
      K), scaled to all M rows).  The whole C and qmat would take
      4 M^2 x 8 bytes of host memory (137 GB at 256 x 256).

    The fused program's value is wrong for K > 240 (the running C is summed
    once per K block, gemm_kernel.h:378-407); its time is not."""

    def __init__(self, name: str, spins: np.ndarray, target_s: float = 1.0):
        orc = _orc()
        w = WORKLOADS[name]
        self.N, self.nf = w["N"], w["nfile"]
        self.J1, self.dt = w["J1"], w["dt"]
        self.M, self.K = self.N * self.N, 3 * self.nf
        self.spins = spins
        self.target_s = target_s
        self.fusion = orc.RefLib("fusion") if orc.RefLib.available("fusion") else None
        self.gemm = orc.RefLib("gemm") if orc.RefLib.available("gemm") else None
        self.threads = 0
        self.llg_replicas = None
        self.rows = {}
        if self.fusion is not None:
            self._size()

    def available(self) -> bool:
        return self.fusion is not None

    def _size(self):
        """Sample sizes for about target_s of host time per part."""
        f = self.fusion
        nf0 = min(self.nf, max(1, int(2e5 / self.M)))
        self.threads = f.setup(self.N, nf0, J1=self.J1, dt=self.dt, threads=0)
        t = f.step_time(self.spins[:nf0])
        self.llg_replicas = int(min(self.nf, max(1, nf0 * self.target_s / max(t, 1e-6))))
        f.setup(self.N, self.nf, J1=self.J1, dt=self.dt, threads=0)
        rows = min(self.M, 256)
        f.fusion_init(self.spins, rows)
        _, _, tb = f.fusion_sqt_timed(self.spins)
        rows = int(min(self.M, max(256, rows * self.target_s / max(tb, 1e-6))))
        self.rows["fused_avx2"] = max(256, rows - rows % 256)
        f.fusion_init(self.spins, self.rows["fused_avx2"])
        if self.gemm is not None:
            self.gemm.setup(self.N, self.nf, J1=self.J1, dt=self.dt, threads=0)
            r0 = min(self.M, 256)
            _, _, tb = self.gemm.gemm_sqt_band(self.spins, self.spins, r0)
            rows = int(min(self.M, max(256, r0 * self.target_s / max(tb, 1e-6))))
            self.rows["openblas"] = max(256, rows - rows % 256)

    def sample(self) -> dict:
        """One bounded sample of one step of each program: seconds per full
        step, extrapolated as described above."""
        f = self.fusion
        f.setup(self.N, self.llg_replicas, J1=self.J1, dt=self.dt, threads=0)
        t_llg = f.step_time(self.spins[:self.llg_replicas]) * self.nf / self.llg_replicas
        f.setup(self.N, self.nf, J1=self.J1, dt=self.dt, threads=0)
        out = {}
        _, tp, tb = f.fusion_sqt_timed(self.spins)
        out["fused_avx2"] = (t_llg, tp + tb * self.M / self.rows["fused_avx2"])
        if self.gemm is not None:
            self.gemm.setup(self.N, self.nf, J1=self.J1, dt=self.dt, threads=0)
            _, tp, tb = self.gemm.gemm_sqt_band(self.spins, self.spins, self.rows["openblas"])
            out["openblas"] = (t_llg, tp + tb * self.M / self.rows["openblas"])
        return out

    def describe(self, path: str, t_llg: float, t_sqt: float) -> dict:
        M, nf, K = self.M, self.nf, self.K
        rows = self.rows[path]
        prog = ("fused-AVX2 program (fused_dgemm)" if path == "fused_avx2"
                else "OpenBLAS program (cblas_dgemm)")
        sample = (f"reference {prog}: runge_kutta+renorm on {self.llg_replicas} of {nf} replicas "
                  f"scaled x{nf / self.llg_replicas:.2f}; S(q,t) A pack whole + GEMM/epilogue on "
                  f"{rows} of {M} rows scaled x{M / rows:.2f}; {self.threads} OpenMP threads")
        d = {"value": M * nf / (t_llg + t_sqt), "unit": "site-steps/s", "cores": self.threads,
             "kind": "reference", "sample": sample,
             "llg_site_steps_per_s": M * nf / t_llg,
             "sqt_tflops": 2.0 * M * M * K / t_sqt / 1e12, "ms_per_step": (t_llg + t_sqt) * 1e3}
        if path == "fused_avx2" and K > 240:
            d["value_valid"] = False
            d["note"] = ("time only: the fused program's S(q,t) is wrong for K > 240 "
                         "(sum taken once per K block)")
        return d

    def close(self):
        if self.fusion is not None:
            self.fusion.lib.ref_fusion_free()


def cpu_baseline_line(name: str, spins: np.ndarray, samples: int = 1, target_s: float = 1.0):
    """The reference's programs, `samples` samples each (median); returns
    (cpu_baseline dict of the faster program, all paths) or (None, None)."""
    ref = CpuReference(name, spins, target_s)
    if not ref.available():
        return None, None
    runs = [ref.sample() for _ in range(samples)]
    paths = {}
    for path in runs[0]:
        t_llg = statistics.median(r[path][0] for r in runs)
        t_sqt = statistics.median(r[path][1] for r in runs)
        paths[path] = ref.describe(path, t_llg, t_sqt)
    ref.close()
    best = max(paths.values(), key=lambda d: d["value"])
    return {k: best[k] for k in ("value", "unit", "cores", "kind", "sample")}, paths


def run_reference(args):
    """--impl reference: the reference's CPU programs on the host cores, each
    step a bounded sample of the workload; `value` is the faster program's.
    Under torchrun rank 0 alone runs; the other ranks exit without work."""
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    name = args.workload
    w = WORKLOADS[name]
    N, nf = w["N"], w["nfile"]
    import asd_b200 as asd

    spins = asd.random_spins(N, nf, seed=0)
    ref = CpuReference(name, spins, target_s=args.ref_target_s)
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libref_fusion.so not built (make -C oracle ref REF=...)"}))
        return 0
    runs = []
    for it in range(args.warmup + args.steps):
        r = ref.sample()
        if it >= args.warmup:
            runs.append(r)
    paths = {}
    for path in runs[0]:
        t_llg = statistics.median(r[path][0] for r in runs)
        t_sqt = statistics.median(r[path][1] for r in runs)
        paths[path] = ref.describe(path, t_llg, t_sqt)
    ref.close()
    best = max(paths.values(), key=lambda d: d["value"])
    value = best["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "site-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": N * N * nf / value * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded spins uniform on the sphere",
        "config": bench_config(name, args),
        "cpu_baseline": {k: best[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": value, "unit": "site-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "paths": paths,
    }
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------- GPU arm
def traffic_for(kernel_key: str):
    """DRAM bytes per launch of a kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None, None
    d = json.loads(p.read_text())
    e = d.get(kernel_key)
    if isinstance(e, dict):
        return e.get("bytes"), e.get("source")
    return e, None


def run_ours(args):
    import torch
    import torch.distributed as dist

    import asd_b200 as asd

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=120))
    name = args.workload
    w = WORKLOADS[name]
    N, nf = w["N"], w["nfile"]
    M, K = N * N, 3 * nf
    mode = args.mode or w["mode"]
    params = asd.Params.make(N, nf, J1=w["J1"], J2=w["J2"], alpha=w["alpha"], h=w["h"], dt=w["dt"])
    asd.load().asd_set_device(local)
    extras = not args.no_extras
    ctx = asd.Context(params, modes=(["fp64", "tf32x3", "bf16x3", "fp16x3"] if extras else [mode]))
    ctx.set_llg_kernel(args.llg_kernel)
    if args.chunk_k >= 0:
        ctx.set_chunk_k(args.chunk_k)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    spins0 = asd.random_spins(N, nf, seed=rank_seed(rank))
    ctx.set_spins(spins0, as_origin=True)
    total = args.warmup + args.steps
    d_out = torch.zeros(2 * max(total, 1), dtype=torch.float64, device="cuda")

    def one_step(i):
        ctx.step(1)
        n1 = ctx.last_launches()
        ctx.sqt_async(mode, d_out.data_ptr() + 16 * i)
        return n1 + ctx.last_launches()

    # kernels timed alone, before the long GEMM loop heats the part: the FP64
    # peaks and each LLG kernel (their roofline denominators are burst figures)
    pre = pre_measurements(ctx, asd, torch, stream, name, args) if (rank == 0 and extras) else {}
    ctx.time_kernels(True)
    for i in range(args.warmup):
        one_step(i)
    torch.cuda.synchronize()
    ctx.kernel_time("gemm")  # forget the warm-up launches
    ctx.kernel_time("llg")
    if world > 1:
        dist.barrier()
    launches = 0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for i in range(args.warmup, total):
            launches += one_step(i)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    gemm_ms, gemm_n = ctx.kernel_time("gemm")
    ctx.kernel_time("llg")  # recorded but not reported: behind a split GEMM the RK4 step
    ctx.time_kernels(False)  # is launched early and its events include the wait for SMs
    ctx.check_device_status()
    ms, value = aggregate(ms, M * nf, world, dist if world > 1 else None, "cuda")
    if world > 1:
        dist.barrier()
    sqt_last = complex(*d_out[2 * (total - 1):2 * total].tolist())

    report = {}
    if rank == 0 and extras:
        report = component_measurements(ctx, asd, torch, stream, name, mode, args, pre)
    e2e = e2e_measurement(ctx, asd, torch, spins0, mode, M, nf, args, world) if extras else None
    if world > 1:
        dist.barrier()
    if rank != 0:
        ctx.close()
        if world > 1:
            dist.destroy_process_group()
        return 0

    peaks = measured_peaks()
    gemm_flops = 2.0 * M * M * K
    gemm_avg_ms = gemm_ms / gemm_n if gemm_n else None
    achieved = gemm_flops / (gemm_avg_ms / 1e3) / 1e12 if gemm_avg_ms else None
    frac = achieved / peaks["bf16_sustained"] if achieved is not None else None
    traffic, traffic_src = traffic_for(f"umma_sqt_{mode}_{N}x{N}x{nf}")
    roofline = {
        "bound": "tensor", "kernel": f"umma_sqt_kernel ({mode})", "achieved": achieved,
        "peak": peaks["bf16_sustained"], "unit": "TFLOP/s", "frac": frac, "traffic": traffic,
        "peak_source": f"{peaks['source']}, dense bf16 sustained (the GEMM runs back to back "
                       f"for the whole timed region)",
        "achieved_counts": "useful 2*M*M*K per launch / mean launch time by CUDA events on the "
                           "GEMM's stream inside the timed region; the 3-term split issues 3x "
                           "that on the tensor pipe",
        "launches_timed": gemm_n, "ms_per_launch": gemm_avg_ms,
        "algorithmic_operand_bytes": 4 * M * (K + (-K) % 64) * (2 if mode == "bf16x3" else 4),
        "traffic_source": traffic_src,
        **split_ceiling(mode, frac),
    }
    if mode == "fp64" and achieved is not None:
        roofline.update({"bound": "fp64 tensor", "kernel": "dmma_sqt_kernel (fp64)"})
    line = {
        "metric": METRIC, "value": value, "unit": "site-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": f"f64 RK4 + {mode} GEMM (fp32 accumulate, f64 reduction)",
        "data": "synthetic: seeded spins uniform on the sphere",
        "config": bench_config(name, args),
        "roofline": roofline,
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "e2e": e2e,
        "timed_region_s": ms * args.steps / 1e3,
        "sqt_last": [sqt_last.real, sqt_last.imag],
    }
    line.update(report)
    if world == 1 and extras and not args.no_cpu_baseline:
        base, paths = cpu_baseline_line(name, spins0, samples=1, target_s=1.0)
        if base is not None:
            line["cpu_baseline"] = base
            line["cpu_baseline_paths"] = paths
    print(json.dumps(line))
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def pre_measurements(ctx, asd, torch, stream, name, args):
    """Rank 0, before the timed region: the FP64 peaks of this GPU and each LLG
    kernel alone (median of 3 runs of 10 steps), timed by CUDA events."""
    fma_tf, _ = asd.measure_fp64_peak("fma", stream.cuda_stream)
    dmma_tf, _ = asd.measure_fp64_peak("dmma", stream.cuda_stream)
    fma_sus, fma_clk = sustained_fma_peak(asd, stream, torch.cuda.current_device())
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 10
    llg, llg_clocks = {}, {}
    for kern in ("stages", "fused"):
        ctx.set_llg_kernel(kern)
        ctx.step(2)
        ts = []
        with ClockSampler(torch.cuda.current_device()) as clk:
            for _ in range(3):
                torch.cuda.synchronize()
                ev0.record(stream)
                ctx.step(reps)
                ev1.record(stream)
                torch.cuda.synchronize()
                ts.append(ev0.elapsed_time(ev1) / reps)
        llg[kern] = sorted(ts)[1]
        llg_clocks[kern] = clk.summary()
    ctx.set_llg_kernel(args.llg_kernel)
    return {"fma_tf": fma_tf, "dmma_tf": dmma_tf, "fma_sustained_tf": fma_sus,
            "fma_sustained_clocks": fma_clk, "llg": llg, "llg_clocks": llg_clocks}


def component_measurements(ctx, asd, torch, stream, name, mode, args, pre):
    """Rank 0, after the timed region: every S(q,t) mode alone (its GEMM
    kernel by CUDA events on its own stream), the split modes' error against
    the FP64 path relative to |S| and to the magnitude of the summed terms;
    with the FP64 peaks and LLG kernels measured before the timed region."""
    w = WORKLOADS[name]
    N, nf = w["N"], w["nfile"]
    M, K = N * N, 3 * nf
    peaks = measured_peaks()
    fma_tf, dmma_tf, llg = pre["fma_tf"], pre["dmma_tf"], pre["llg"]
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    d = torch.zeros(2, dtype=torch.float64, device="cuda")
    sqt_ms, kern_ms, vals = {}, {}, {}
    ctx.time_kernels(True)
    for m in ("fp64", "tf32x3", "bf16x3", "fp16x3"):
        n = 1 if m == "fp64" else 3
        ctx.sqt_async(m, d.data_ptr())  # operands split, warm
        torch.cuda.synchronize()
        ctx.kernel_time("gemm")
        ev0.record(stream)
        for _ in range(n):
            ctx.sqt_async(m, d.data_ptr())
        ev1.record(stream)
        torch.cuda.synchronize()
        sqt_ms[m] = ev0.elapsed_time(ev1) / n
        km, kn = ctx.kernel_time("gemm")
        kern_ms[m] = km / kn if kn else None
        vals[m] = complex(*d.tolist())
    ctx.time_kernels(False)
    mag = ctx.sqt_magnitude()
    ref = vals["fp64"]
    flops = 2.0 * M * M * K
    sqt = {}
    for m in sqt_ms:
        e = {"ms": sqt_ms[m], "gemm_kernel_ms": kern_ms[m],
             "tflops": flops / (sqt_ms[m] / 1e3) / 1e12,
             "value": [vals[m].real, vals[m].imag],
             "rel_err_vs_fp64": abs(vals[m] - ref) / abs(ref),
             "err_vs_fp64_rel_to_term_magnitude": abs(vals[m] - ref) / mag}
        if m == "fp64":
            e["fp64_dmma_peak_tflops"] = dmma_tf
            e["frac_of_fp64_dmma_peak"] = (flops / (kern_ms[m] / 1e3) / 1e12 / dmma_tf
                                           if kern_ms[m] else None)
            e["peak_note"] = ("the peak is a ~1 ms burst before the timed region; this GEMM runs "
                              "for most of a second after it, under the power cap")
        sqt[m] = e
    return {
        "fp64_peaks": {"fma_tflops": fma_tf, "fma_tops": fma_tf / 2.0, "dmma_tflops": dmma_tf,
                       "source": "asd_measure_fp64_peak on this GPU before the timed region "
                                 "(burst, ~1 ms each)",
                       "fma_sustained_tflops": pre.get("fma_sustained_tf"),
                       "fma_sustained_clocks": pre.get("fma_sustained_clocks"),
                       "sustained_source": "the FMA peak kernel back to back for 0.3 s"},
        "llg": add_per_clock(
            llg_report(llg, M * nf, llg_fp64_ops(w["J2"] != 0.0, any(w["h"]), w["alpha"] != 0.0),
                       peaks["hbm_gbs"], fma_tf / 2.0,
                       (pre["fma_sustained_tf"] / 2.0) if pre.get("fma_sustained_tf") else None),
            pre.get("llg_clocks"), pre.get("fma_sustained_clocks")),
        "llg_note": "each LLG kernel alone before the timed region (median of 3 x 10 steps)",
        "llg_clocks": pre.get("llg_clocks"),
        "sqt": sqt,
        "sqt_term_magnitude": mag,
        "sqt_speedup_vs_fp64": {m: sqt_ms["fp64"] / sqt_ms[m]
                                for m in ("tf32x3", "bf16x3", "fp16x3")},
    }


def e2e_measurement(ctx, asd, torch, spins0, mode, M, nf, args, world):
    """End to end through the host-buffer API, per step: pinned host spins in,
    RK4 + S(q,t), spins and S(q,t) back to pinned host memory (each step's
    input is the previous step's output).  The headline form enqueues the
    steps with asd_ctx_step_host_async, so consecutive steps overlap chunk by
    chunk, and synchronises once at the end; the synchronous
    asd_ctx_step_host (one call = one complete step) is reported beside it."""
    import torch.distributed as dist

    n = M * nf * 3
    h_in = torch.from_numpy(spins0.reshape(-1).copy()).pin_memory()
    h_out = torch.empty(n, dtype=torch.float64).pin_memory()
    steps = max(2, min(args.steps, 10))
    h_sqt = torch.zeros(2 * steps, dtype=torch.float64).pin_memory()
    ctx.step_host(h_in.data_ptr(), h_out.data_ptr(), mode)  # warm
    t0 = time.perf_counter()
    for _ in range(steps):
        ctx.step_host(h_out.data_ptr(), h_out.data_ptr(), mode)
    ms_sync = (time.perf_counter() - t0) / steps * 1e3
    ctx.step_host_async(h_out.data_ptr(), h_out.data_ptr(), mode, h_sqt.data_ptr())  # warm
    ctx.synchronize()
    t0 = time.perf_counter()
    for i in range(steps):
        ctx.step_host_async(h_out.data_ptr(), h_out.data_ptr(), mode, h_sqt.data_ptr() + 16 * i)
    ctx.synchronize()
    ms = (time.perf_counter() - t0) / steps * 1e3
    # the floor: the same bytes up and down at once on two streams, no compute
    d_a = torch.empty(n, dtype=torch.float64, device="cuda")
    d_b = torch.empty(n, dtype=torch.float64, device="cuda")
    s_up, s_down = torch.cuda.Stream(), torch.cuda.Stream()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(3):
        with torch.cuda.stream(s_up):
            d_a.copy_(h_in, non_blocking=True)
        with torch.cuda.stream(s_down):
            h_out.copy_(d_b, non_blocking=True)
    torch.cuda.synchronize()
    copy_ms = (time.perf_counter() - t0) / 3 * 1e3
    del d_a, d_b
    ms, value = aggregate(ms, M * nf, world, dist if world > 1 else None, "cuda")
    ms_sync, value_sync = aggregate(ms_sync, M * nf, world, dist if world > 1 else None, "cuda")
    return {"value": value, "unit": "site-steps/s", "h2d_bytes_per_step": n * 8,
            "d2h_bytes_per_step": n * 8 + 16, "ms_per_step": ms, "steps": steps,
            "api": "asd_ctx_step_host_async x steps + asd_ctx_synchronize (pinned host buffers)",
            "copy_bound_ms_per_step": copy_ms, "frac_of_copy_bound": copy_ms / ms,
            "copy_bound": "the step's bytes up and down at once on two streams, no compute",
            "sync": {"value": value_sync, "ms_per_step": ms_sync,
                     "api": "asd_ctx_step_host (pinned host buffers)"}}


# ------------------------------------------------------ other configurations
def timed(torch, fn, reps):
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(reps):
        fn()
    e1.record(s)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def run_secondary(args):
    """Secondary workloads, one JSON line each (not the headline):
    grid32   32x32 lattice, 200 replicas, 2000 steps, FP64, S(q,t) on the whole q
             grid after every step
    adjoint64  64x64 lattice, 100 replicas, 1000 steps, S(q,t) every 10 steps,
             checkpoints every 50: loss + gradient wrt (J1, J2, alpha, h)
    batch48  48 lattices of sizes in {48,64,96,128,160}^2, noise amplitude in
             [0, 0.5], alpha in [0.01, 0.2]: 2000 steps in one persistent launch
    grid128, grid256  S(q,t) on the whole q grid after one step of the 128x128x500
             and 256x256x1000 workloads, every mode, against one q of the same mode
    llg128j2, llg256j2  the LLG kernels alone on the 128x128 lattice with 500
             replicas or the 256x256 lattice with 1000, with the 256x256
             workload's model (J=1, J2=-0.3, alpha=0.02): stage kernels against
             HBM, the one-launch step against FP64 issue"""
    import torch

    import asd_b200 as asd

    torch.cuda.set_device(0)
    out = {"impl": "ours", "workload": args.workload, "n_gpus": 1, "data": "synthetic"}
    if args.workload in ("grid128", "grid256"):
        w = WORKLOADS["sqt128" if args.workload == "grid128" else "sqt256"]
        N, nf = w["N"], w["nfile"]
        M, K = N * N, 3 * nf
        ctx = asd.Context(asd.Params.make(N, nf, J1=w["J1"], J2=w["J2"], alpha=w["alpha"],
                                          h=w["h"], dt=w["dt"]))
        stream = torch.cuda.current_stream()
        ctx.set_stream(stream.cuda_stream)
        ctx.set_spins(asd.random_spins(N, nf, seed=0), as_origin=True)
        ctx.step(1)
        grid = torch.zeros(2 * M, dtype=torch.float64, device="cuda")
        one = torch.zeros(2, dtype=torch.float64, device="cuda")
        res = {}
        for mode in ("bf16x3", "fp16x3", "tf32x3", "fp64"):
            reps = 1 if mode == "fp64" else 3
            ctx.sqt_grid_async(mode, grid.data_ptr())  # work space, warm
            g_ms = timed(torch, lambda: ctx.sqt_grid_async(mode, grid.data_ptr()), reps)
            ctx.sqt_async(mode, one.data_ptr())
            q_ms = timed(torch, lambda: ctx.sqt_async(mode, one.data_ptr()), reps)
            g = grid.view(N, N, 2)
            vx = N // 10
            res[mode] = {"grid_ms": g_ms, "single_q_ms": q_ms, "grid_over_single": g_ms / q_ms,
                         "gemm_tflops": 2.0 * M * M * K / (g_ms / 1e3) / 1e12,
                         "grid_at_vx_vy": [float(g[vx, vx, 0]), float(g[vx, vx, 1])],
                         "single_q": one.tolist()}
        out.update({
            "metric": "S(q,t) on the whole N x N q grid, ms per evaluation", "unit": "ms",
            "value": res[w["mode"]]["grid_ms"], "higher_is_better": False,
            "dtype": w["mode"] + " GEMM, f64 bins and DFT",
            "config": {"workload": w["desc"] + ", S(q,t) at all N*N q", "sites": M, "replicas": nf},
            "modes": res,
        })
        ctx.close()
    elif args.workload in ("llg128j2", "llg256j2"):
        N, nf = (128, 500) if args.workload == "llg128j2" else (256, 1000)
        M = N * N
        ctx = asd.Context(asd.Params.make(N, nf, J1=1.0, J2=-0.3, alpha=0.02, dt=0.005),
                          modes=["fp64"])
        stream = torch.cuda.current_stream()
        ctx.set_stream(stream.cuda_stream)
        ctx.set_spins(asd.random_spins(N, nf, seed=0), as_origin=True)
        fma_tf, _ = asd.measure_fp64_peak("fma", stream.cuda_stream)
        fma_sus, fma_clk = sustained_fma_peak(asd, stream, 0)
        llg_ms, llg_clk = {}, {}
        for kern in ("stages", "fused"):
            ctx.set_llg_kernel(kern)
            ctx.step(3)
            with ClockSampler(0) as clk:
                llg_ms[kern] = timed(torch, lambda: ctx.step(1), max(args.steps, 10))
            llg_clk[kern] = clk.summary()
        out.update({
            "metric": "LLG site-steps/s (RK4 step alone)", "unit": "site-steps/s",
            "value": M * nf / (llg_ms["fused"] / 1e3), "higher_is_better": True,
            "dtype": "f64",
            "config": {"workload": f"{N}x{N} lattice, {nf} replicas, J=1, J2=-0.3, alpha=0.02, "
                                   "dt=0.005, RK4 step only", "sites": M, "replicas": nf},
            "llg": add_per_clock(llg_report(llg_ms, M * nf, llg_fp64_ops(True, False, True),
                                            measured_peaks()["hbm_gbs"], fma_tf / 2.0,
                                            fma_sus / 2.0), llg_clk, fma_clk),
            "llg_clocks": llg_clk, "fma_sustained_clocks": fma_clk,
        })
        ctx.close()
    elif args.workload == "grid32":
        # 32x32 lattice, 200 replicas, J=1, alpha=0.1, dt=0.01, 2000 RK4 steps, S(q,t) on the
        # whole 32x32 q grid after every step (FP64 GEMM + displacement bins + 2-D DFT)
        N, nf, nsteps = 32, 200, 2000
        M = N * N
        ctx = asd.Context(asd.Params.make(N, nf, J1=1.0, alpha=0.1, dt=0.01), modes=["fp64"])
        stream = torch.cuda.current_stream()
        ctx.set_stream(stream.cuda_stream)
        ctx.set_spins(asd.random_spins(N, nf, seed=0), as_origin=True)
        grid = torch.zeros(2 * M * nsteps, dtype=torch.float64, device="cuda")

        def run(n):
            for i in range(n):
                ctx.step(1)
                ctx.sqt_grid_async("fp64", grid.data_ptr() + 16 * M * i)

        run(5)
        ms = timed(torch, lambda: run(nsteps), 1) / nsteps
        step_ms = timed(torch, lambda: ctx.step(1), 200)
        out.update({
            "metric": "RK4 steps with the full-q-grid S(q,t) per second (FP64)",
            "value": 1e3 / ms, "unit": "steps/s", "higher_is_better": True,
            "ms_per_step": ms, "dtype": "f64", "site_steps_per_s": M * nf / (ms / 1e3),
            "config": {"workload": "32x32 lattice, 200 replicas, J=1, alpha=0.1, dt=0.01, "
                                   "2000 steps, S(q,t) on the 32x32 q grid every step",
                       "sites": M, "replicas": nf},
            "llg_ms_per_step": step_ms,
            "sqt_grid_ms": ms - step_ms,
            "l2": "the whole state (4.9 MB) is L2-resident: not an HBM measurement",
        })
        ctx.close()
    elif args.workload == "adjoint64":
        N, nf, nsteps, stride, ck = 64, 100, 1000, 10, 50
        s0 = asd.random_spins(N, nf, seed=0)
        ctx = asd.Context(asd.Params.make(N, nf, J1=1.0, alpha=0.1, h=(0, 0, 0.2), dt=0.01),
                          modes=["fp64"])
        ctx.set_spins(s0, as_origin=True)
        _, _, target = ctx.loss_grad(nsteps, stride, ck, None)
        ctx.set_params(asd.Params.make(N, nf, J1=0.8, alpha=0.15, dt=0.01))
        t0 = time.perf_counter()
        fwd = ctx.loss_grad(nsteps, stride, ck, None)
        t_fwd = time.perf_counter() - t0
        t0 = time.perf_counter()
        loss, grad, _ = ctx.loss_grad(nsteps, stride, ck, target)
        t_grad = time.perf_counter() - t0
        out.update({
            "metric": "loss + adjoint gradient wall time", "value": t_grad, "unit": "s",
            "higher_is_better": False,
            "config": {"workload": "64x64 lattice, 100 replicas, 1000 steps, S(q,t) every 10 steps, checkpoints every 50"},
            "forward_only_s": t_fwd, "loss": loss, "grad": list(grad),
            "site_steps_per_s_forward": N * N * nf * nsteps / t_fwd,
        })
        ctx.close()
    elif args.workload == "batch48":
        rng = np.random.default_rng(5)
        sizes = [int(x) for x in rng.choice([48, 64, 96, 128, 160], size=48)]
        lats = []
        for k, N in enumerate(sizes):
            lats.append(asd.Lattice.make(N, J1=1.0, alpha=float(rng.uniform(0.01, 0.2)), dt=0.01))
        b = asd.Batch(lats)
        for l, N in enumerate(sizes):
            b.set_spins(l, asd.noisy_ordered_spins(N, float(rng.uniform(0, 0.5)), l).astype(np.float32))
        if args.batch_cluster:
            b.configure_cluster(args.batch_cluster, 0)
            tile, ctas = 0, args.batch_cluster
        else:
            tile, ctas, _ = b.autotune(20)

        def time_run(n=2000):
            b.run(10)
            t0 = time.perf_counter()
            b.run(n)
            return time.perf_counter() - t0

        t = time_run()
        sites = sum(N * N for N in sizes)
        chosen = ({"kernel": "cluster-resident", "cluster_size": ctas} if tile == 0 else
                  {"kernel": "global-memory", "tile": tile, "ctas_per_sm": ctas})
        # the other kernel family, for comparison (its autotuned best is not kept)
        if tile == 0:
            b.configure(256, 4)
            other = {"kernel": "global-memory", "tile": 256, "ctas_per_sm": 4}
        else:
            try:
                b.configure_cluster(8, 512)
                other = {"kernel": "cluster-resident", "cluster_size": 8}
            except asd.AsdError:
                other = None
        if other is not None:
            other["ms_per_step"] = time_run() / 2000 * 1e3
        out.update({
            "metric": "batched site-steps/s (one persistent launch, 2000 steps)",
            "value": sites * 2000 / t, "unit": "site-steps/s", "ms_per_step": t / 2000 * 1e3,
            "dtype": "f32 RK4 + f64 renorm",
            "config": {"workload": "48 lattices, sizes in {48,64,96,128,160}^2", "sites": sites,
                       **chosen},
            "other_kernel": other,
        })
        b.close()
    print(json.dumps(out))
    return 0


def run_sharded(args):
    """--shard: the workload's one ensemble split by replicas over the ranks --
    strong scaling of one system.  Each rank steps its
    replicas; every step's S(q,t) is exchanged through asd_b200.shard
    (all-reduces of 2 and 3*N*N doubles over NCCL) and is the same on every
    rank.  Device-resident: no e2e leg."""
    import torch
    import torch.distributed as dist

    import asd_b200 as asd
    from asd_b200.shard import ShardedSqt, shard_range

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=120))
    w = WORKLOADS[args.workload]
    N, nf = w["N"], w["nfile"]
    M = N * N
    b, e = shard_range(nf, rank, world)
    mode = args.mode or w["mode"]
    params = asd.Params.make(N, e - b, J1=w["J1"], J2=w["J2"], alpha=w["alpha"], h=w["h"],
                             dt=w["dt"])
    asd.load().asd_set_device(local)
    ctx = asd.Context(params, modes=[mode])
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    ctx.set_spins(asd.random_spins(N, nf, seed=0)[b:e], as_origin=True)  # one ensemble
    ens = ShardedSqt(ctx, nf, M)
    ens.exchange_origin()
    total = args.warmup + args.steps
    d_out = torch.zeros(2 * max(total, 1), dtype=torch.float64, device="cuda")

    def one_step(i):
        ctx.step(1)
        n = ctx.last_launches()
        ens.sqt_async(mode, d_out[2 * i:2 * i + 2])
        return n + ens.launches

    for i in range(args.warmup):
        one_step(i)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = 0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for i in range(args.warmup, total):
            launches += one_step(i)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    ctx.check_device_status()
    # units per rank = its share of the one ensemble, so the sum over ranks is the ensemble
    ms, value = aggregate(ms, M * nf / world, world, dist if world > 1 else None, "cuda")
    sqt_last = complex(*d_out[2 * (total - 1):2 * total].tolist())
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": "site-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": f"f64 RK4 + {mode} GEMM (fp32 accumulate, f64 reduction)",
        "data": "synthetic: seeded spins uniform on the sphere",
        "config": {**bench_config(args.workload, args),
                   "workload": w["desc"] + ", one ensemble split by replicas",
                   "parallelism": f"replicas/{world}", "exchange_doubles_per_step": 2 + 3 * M},
        "gpu_launches": launches, "clocks": clk.summary(), "e2e": None,
        "sqt_last": [sqt_last.real, sqt_last.imag],
    }))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["sqt256", "sqt128", "grid32", "grid128", "grid256",
                                           "adjoint64", "batch48", "llg128j2", "llg256j2"],
                    default="sqt256",
                    help="sqt256 (default) and sqt128 print the full line; the others a line of "
                         "their own")
    ap.add_argument("--mode", choices=["tf32x3", "bf16x3", "fp16x3", "fp64"], default=None,
                    help="S(q,t) arithmetic (default: the workload's)")
    ap.add_argument("--batch-cluster", type=int, default=0,
                    help="batch48: clusters of this many CTAs instead of the autotuner's choice")
    ap.add_argument("--llg-kernel", choices=["auto", "fused", "stages"], default="auto",
                    help="RK4 step: one streamed launch where it fills the GPU (auto, default), "
                         "always (fused) or four stage kernels (stages)")
    ap.add_argument("--chunk-k", type=int, default=-1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="only the timed steps (for profiling): one S(q,t) mode allocated, no "
                         "per-component timings, e2e or CPU baseline")
    ap.add_argument("--ref-target-s", type=float, default=0.5,
                    help="--impl reference: host seconds per sampled part of a step")
    ap.add_argument("--shard", action="store_true",
                    help="strong scaling: split the workload's one ensemble by replicas over the "
                         "ranks (S(q,t) exchanged every step) instead of one ensemble per rank")
    args = ap.parse_args()
    if args.workload not in WORKLOADS:
        return run_secondary(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.shard:
        return run_sharded(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
