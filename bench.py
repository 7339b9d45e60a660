#!/usr/bin/env python
"""Benchmark of the hot path: one RK4 step of the LLG equation for every
replica plus one S(q,t) evaluation, on the 128 x 128 lattice with 500
replicas (antiferromagnetic J = -1, h = (0, 0, 0.5), alpha = 0.05,
dt = 0.005), the correlation GEMM in TF32x3.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line on rank 0.  ``value`` is the whole job's throughput in
site-steps/s (a site-step = one spin of one replica advanced one RK4 step,
with the step's S(q,t) evaluation included), with the spins resident in HBM.
``e2e`` is the same metric through asd_ctx_step_host: the spins come from
pinned host memory and go back every step, as the reference's runge_kutta
contract has them.  Under torchrun every rank runs its own lattice (weak
scaling, no collective in the data path); the time is the max over ranks.

``--impl reference`` times the reference's own C code (oracle/_ref, compiled
from its sources) on the host cores: runge_kutta + renormalisation on the full
lattice and fused_dgemm's S(q,t) on a band of rows, scaled to the full
lattice.
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

CONFIG = dict(N=128, nfile=500, J1=-1.0, J2=0.0, alpha=0.05, h=(0.0, 0.0, 0.5), dt=0.005)
WORKLOAD = "llg-rk4+sqt 128x128 lattice, 500 replicas, J=-1, h=(0,0,0.5), alpha=0.05, dt=0.005"
METRIC = "LLG site-steps/s + S(q,t) GEMM TFLOP/s, mixed vs FP64 plain at stated error"
LLG_BYTES_PER_SITE_STEP = 384  # 4 fused stage kernels: 3+5+5+3 FP64 3-vectors
LLG_FUSED_BYTES_PER_SITE_STEP = 48  # one streamed step: read y, write y


def llg_fp64_ops(J2: bool, H: bool, damp: bool) -> int:
    """FP64 operations of one site-step as the kernels write them (add, sub,
    mul and fma 1 each; a division or square root 1 each, although the
    hardware runs a short sequence for them): the right-hand side (exchange
    12 mul + 12 add, J2 as much again, the field 3 add, H x S 9, damping 18)
    and dt * f (3) in each of the 4 stages, then the stage combinations
    (18 + 18 + 15) and stage 4's combination and renormalisation (24)."""
    rhs = 24 + (24 if J2 else 0) + (3 if H else 0) + 9 + (18 if damp else 0)
    return 4 * (rhs + 3) + 18 + 18 + 15 + 24


def fp64_peak_tops(torch) -> float:
    """Nominal FP64 issue rate: 64 FP64 lanes per SM per clock at the maximum
    SM clock (1 operation per lane per clock; no measured FP64 figure exists)."""
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    mhz = 1965.0
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        mhz = json.loads(p.read_text()).get("sm_max_mhz", mhz)
    return sms * 64 * mhz * 1e6 / 1e12


def llg_report(ms_by_kernel, sites_replicas, ops, hbm, fp64_peak):
    """Per LLG kernel: site-steps/s, DRAM bytes against the HBM peak (the
    bound of the stage kernels) and FP64 operations against the FP64 issue
    rate (the bound of the one-launch step)."""
    out = {}
    for k, ms in ms_by_kernel.items():
        bps = LLG_BYTES_PER_SITE_STEP if k == "stages" else LLG_FUSED_BYTES_PER_SITE_STEP
        rate = sites_replicas / (ms / 1e3)
        out[k] = {"site_steps_per_s": rate, "ms": ms, "bytes_per_site_step": bps,
                  "achieved_gbs": bps * rate / 1e9, "hbm_peak_gbs": hbm,
                  "frac": bps * rate / 1e9 / hbm, "fp64_ops_per_site_step": ops,
                  "achieved_fp64_tops": ops * rate / 1e12, "fp64_peak_tops_nominal": fp64_peak,
                  "fp64_frac": ops * rate / 1e12 / fp64_peak,
                  "bound": "hbm" if k == "stages" else "fp64"}
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


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def split_ceiling(mode, frac):
    """The highest useful-flop fraction of the dense BF16 peak a 3-term split
    GEMM can reach: three tensor-core products per useful one, and TF32
    products run at half the BF16 rate on B200.  frac_of_ceiling is how close
    the kernel is to that bound."""
    ceil = {"tf32x3": 1.0 / 6.0, "bf16x3": 1.0 / 3.0}.get(mode)
    if ceil is None:
        return {}
    return {"split_ceiling_frac": ceil, "frac_of_split_ceiling": frac / ceil}


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
def cpu_reference_sample(N, nfile, J1, dt, spins, target_s=2.0, llg=True):
    """Times the reference's own compiled code (oracle/_ref/libref_fusion.so) on
    the host cores: runge_kutta + renormalisation on the whole lattice, and the
    fused S(q,t) (llg_sqt_fusion.c:370-441 around fused_dgemm) on a band of
    rows, scaled to all rows.  Returns seconds per full step and a description.
    The reference model has no damping or field: its RK4 costs the same
    regardless of those parameters."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc

    if not orc.RefLib.available("fusion"):
        return None
    r = orc.RefLib("fusion")
    threads = r.setup(N, nfile, J1=J1, dt=dt, threads=0)
    M = N * N
    t_llg = 0.0
    if llg:
        s = spins.copy()
        r.steps(s, 1, 1.0)  # warm
        t0 = time.perf_counter()
        s = r.steps(s, 1, 1.0)
        t_llg = time.perf_counter() - t0
    # size the band of GEMM rows so one evaluation takes about target_s
    rows = 256
    r.fusion_init(spins, rows)
    t0 = time.perf_counter()
    r.fusion_sqt(spins)
    t_small = time.perf_counter() - t0
    rows = int(min(M, max(256, rows * target_s / max(t_small, 1e-6))))
    rows -= rows % 256
    rows = max(rows, 256)
    r.fusion_init(spins, rows)
    t0 = time.perf_counter()
    r.fusion_sqt(spins)
    t_band = time.perf_counter() - t0
    r.lib.ref_fusion_free()
    t_sqt = t_band * M / rows
    sample = (f"reference runge_kutta+renorm on all {M}x{nfile} site-replicas, fused_dgemm S(q,t) "
              f"on {rows} of {M} rows scaled by {M / rows:.2f}, {threads} OpenMP threads")
    return dict(t_llg=t_llg, t_sqt=t_sqt, threads=threads, sample=sample, rows=rows)


def cpu_reference_openblas(N, nfile, J1, dt, spins):
    """Times the reference's gemm program (gemm/llg_sqt_mkl.c, compiled from its
    sources into oracle/_ref/libref_gemm.so against the image's OpenBLAS) on the
    host cores: runge_kutta + renormalisation on the whole lattice and its
    S(q,t) -- cblas_dgemm of the whole (N^2 x N^2) correlation matrix, then the
    outer-product subtraction and the phase reduction (gemm/llg_sqt_mkl.c:
    369-423) -- on the full workload.  Returns a cpu_baseline-style dict."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc

    if not orc.RefLib.available("gemm"):
        return None
    r = orc.RefLib("gemm")
    threads = r.setup(N, nfile, J1=J1, dt=dt, threads=0)
    M = N * N
    s = r.steps(spins, 1, 1.0)  # warm
    t0 = time.perf_counter()
    s = r.steps(s, 1, 1.0)
    t_llg = time.perf_counter() - t0
    t0 = time.perf_counter()
    r.gemm_sqt(s, spins)
    t_sqt = time.perf_counter() - t0
    return {"value": M * nfile / (t_llg + t_sqt), "unit": "site-steps/s", "cores": threads,
            "kind": "reference",
            "sample": f"reference gemm program (OpenBLAS cblas_dgemm): runge_kutta+renorm and "
                      f"S(q,t) on all {M}x{nfile} site-replicas, one step, {threads} OpenMP threads",
            "llg_site_steps_per_s": M * nfile / t_llg,
            "sqt_tflops": 2.0 * M * M * 3 * nfile / t_sqt / 1e12}


def run_reference(args):
    """The reference's CPU implementations of the path on the host cores: its
    fused-AVX2 program (fused_dgemm, sampled on a band of rows each step) and
    its OpenBLAS program (full workload, up to 3 samples).  `value` is the
    faster of the two, so the comparison is against the reference's best."""
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    N, nf = CONFIG["N"], CONFIG["nfile"]
    import asd_b200 as asd

    spins = asd.random_spins(N, nf, seed=0)
    vals = []
    info = None
    for it in range(args.warmup + args.steps):
        info = cpu_reference_sample(N, nf, CONFIG["J1"], CONFIG["dt"], spins,
                                    target_s=args.ref_target_s)
        if info is None:
            print(json.dumps({"impl": "reference", "unavailable":
                              "oracle/_ref/libref_fusion.so not built (make -C oracle ref)"}))
            return 0
        if it >= args.warmup:
            vals.append(info["t_llg"] + info["t_sqt"])
    t = statistics.median(vals)
    fused = {"value": N * N * nf / t, "unit": "site-steps/s", "cores": info["threads"],
             "kind": "reference", "sample": info["sample"],
             "llg_site_steps_per_s": N * N * nf / info["t_llg"],
             "sqt_tflops": 2.0 * (N * N) ** 2 * 3 * nf / info["t_sqt"] / 1e12}
    ob = [cpu_reference_openblas(N, nf, CONFIG["J1"], CONFIG["dt"], spins)
          for _ in range(min(max(args.steps, 1), 3))]
    openblas = None
    if ob[0] is not None:
        openblas = sorted(ob, key=lambda d: d["value"])[len(ob) // 2]
    best = fused if openblas is None or fused["value"] >= openblas["value"] else openblas
    value = best["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "site-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": N * N * nf / value * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded spins uniform on the sphere",
        "config": {"workload": WORKLOAD, "sites": N * N, "replicas": nf, "gemm_m": N * N,
                   "gemm_k": 3 * nf},
        "cpu_baseline": {k: best[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": value, "unit": "site-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "paths": {"fused_avx2": fused, "openblas": openblas},
    }
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------- GPU arm
def run_ours(args):
    import torch
    import torch.distributed as dist

    import asd_b200 as asd

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=120))
    N, nf = CONFIG["N"], CONFIG["nfile"]
    M, K = N * N, 3 * nf
    mode = args.mode
    params = asd.Params.make(N, nf, J1=CONFIG["J1"], J2=CONFIG["J2"], alpha=CONFIG["alpha"],
                             h=CONFIG["h"], dt=CONFIG["dt"])
    asd.load().asd_set_device(local)
    ctx = asd.Context(params, modes=["fp64", "tf32x3", "bf16x3"])
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
    ms, value = aggregate(ms, M * nf, world, dist if world > 1 else None, "cuda")
    if world > 1:
        dist.barrier()
    sqt_last = complex(*d_out[2 * (total - 1):2 * total].tolist())

    extra = {"sqt_ms": {}, "report": {}}
    if rank == 0 and not args.no_extras:
        extra = component_measurements(ctx, asd, torch, stream, M, K, nf, args)
    e2e = None if args.no_extras else e2e_measurement(ctx, asd, torch, spins0, mode, M, nf,
                                                      args, world)
    if world > 1:
        dist.barrier()
    if rank != 0:
        ctx.close()
        if world > 1:
            dist.destroy_process_group()
        return 0

    hbm, bf16, src = measured_peaks()
    gemm_flops = 2.0 * M * M * K
    gemm_ms = extra["sqt_ms"].get(mode)  # absent with --no-extras: the GEMM is not timed alone
    achieved = gemm_flops / (gemm_ms / 1e3) / 1e12 if gemm_ms else None
    frac = achieved / bf16 if achieved is not None else None
    traffic = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get(f"umma_sqt_{mode}")
    line = {
        "metric": METRIC, "value": value, "unit": "site-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": f"f64 RK4 + {mode} GEMM (fp32 accumulate, f64 reduction)",
        "data": "synthetic: seeded spins uniform on the sphere",
        "config": {"workload": WORKLOAD, "sites": M, "replicas": nf, "gemm_m": M, "gemm_n": M,
                   "gemm_k": K, "sqt_mode": mode, "llg_kernel": args.llg_kernel,
                   "chunk_k": args.chunk_k if args.chunk_k >= 0 else (512 if mode == "tf32x3" else 1024),
                   "l2": "inputs larger than L2 (spin state 197 MB per array, operands 197 MB)"},
        "roofline": {"bound": "tensor", "kernel": f"umma_sqt_kernel ({mode})",
                     "achieved": achieved, "peak": bf16, "unit": "TFLOP/s",
                     "frac": frac, "traffic": traffic,
                     "peak_source": f"{src} dense bf16 burst (MEASURED_PEAKS.json)",
                     "achieved_counts": "useful 2*M*M*K per evaluation; the 3-term split issues 3x that on the tensor pipe",
                     **(split_ceiling(mode, frac) if frac is not None else {})},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "e2e": e2e,
        "sqt_last": [sqt_last.real, sqt_last.imag],
    }
    line.update(extra["report"])
    if world == 1 and not args.no_cpu_baseline and not args.no_extras:
        # the reference's two CPU programs; cpu_baseline is the faster one
        info = cpu_reference_sample(N, nf, CONFIG["J1"], CONFIG["dt"], spins0, target_s=1.5)
        paths = {}
        if info is not None:
            v = M * nf / (info["t_llg"] + info["t_sqt"])
            paths["fused_avx2"] = {"value": v, "unit": "site-steps/s", "cores": info["threads"],
                                   "kind": "reference", "sample": info["sample"]}
        ob = cpu_reference_openblas(N, nf, CONFIG["J1"], CONFIG["dt"], spins0)
        if ob is not None:
            paths["openblas"] = ob
        if paths:
            best = max(paths.values(), key=lambda d: d["value"])
            line["cpu_baseline"] = {k: best[k] for k in ("value", "unit", "cores", "kind", "sample")}
            line["cpu_baseline_paths"] = paths
    print(json.dumps(line))
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def component_measurements(ctx, asd, torch, stream, M, K, nf, args):
    """LLG alone, every S(q,t) mode alone, and the split modes' error against
    the FP64 path, on the current state (rank 0)."""
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    d = torch.zeros(2, dtype=torch.float64, device="cuda")
    reps = 30
    llg = {}
    for kern in ("stages", "fused"):
        ctx.set_llg_kernel(kern)
        ctx.step(5)
        torch.cuda.synchronize()
        ev0.record(stream)
        ctx.step(reps)
        ev1.record(stream)
        torch.cuda.synchronize()
        llg[kern] = ev0.elapsed_time(ev1) / reps
    ctx.set_llg_kernel(args.llg_kernel)
    hbm, bf16, src = measured_peaks()
    sqt_ms, vals = {}, {}
    for mode in ("fp64", "tf32x3", "bf16x3"):
        n = 2 if mode == "fp64" else 5
        ctx.sqt_async(mode, d.data_ptr())  # operands split, warm
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(n):
            ctx.sqt_async(mode, d.data_ptr())
        ev1.record(stream)
        torch.cuda.synchronize()
        sqt_ms[mode] = ev0.elapsed_time(ev1) / n
        vals[mode] = complex(*d.tolist())
    ref = vals["fp64"]
    flops = 2.0 * M * M * K
    report = {
        "llg": llg_report(llg, M * nf, llg_fp64_ops(CONFIG["J2"] != 0.0, any(CONFIG["h"]),
                                                     CONFIG["alpha"] != 0.0),
                          hbm, fp64_peak_tops(torch)),
        "sqt": {m: {"ms": sqt_ms[m], "tflops": flops / (sqt_ms[m] / 1e3) / 1e12,
                    "value": [vals[m].real, vals[m].imag],
                    "rel_err_vs_fp64": abs(vals[m] - ref) / abs(ref)} for m in sqt_ms},
        "sqt_speedup_vs_fp64": {m: sqt_ms["fp64"] / sqt_ms[m] for m in ("tf32x3", "bf16x3")},
    }
    return {"sqt_ms": sqt_ms, "report": report}


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


def run_workload(args):
    """Secondary workloads, one JSON line each (not the headline):
    grid32   32x32 lattice, 200 replicas, 2000 steps, FP64, S(q,t) on the whole q
             grid after every step
    sqt256   256x256 lattice, 1000 replicas, J=1, J2=-0.3, alpha=0.02, dt=0.005:
             one RK4 step + S(q,t) in BF16x3, with the FP64 path's time and error
    adjoint64  64x64 lattice, 100 replicas, 1000 steps, S(q,t) every 10 steps,
             checkpoints every 50: loss + gradient wrt (J1, J2, alpha, h)
    batch48  48 lattices of sizes in {48,64,96,128,160}^2, noise amplitude in
             [0, 0.5], alpha in [0.01, 0.2]: 2000 steps in one persistent launch"""
    import torch

    import asd_b200 as asd

    torch.cuda.set_device(0)
    hbm, bf16, src = measured_peaks()
    out = {"impl": "ours", "workload": args.workload, "n_gpus": 1, "data": "synthetic"}
    if args.workload == "sqt256":
        N, nf = 256, 1000
        M, K = N * N, 3 * nf
        ctx = asd.Context(asd.Params.make(N, nf, J1=1.0, J2=-0.3, alpha=0.02, dt=0.005),
                          modes=["fp64", "bf16x3", "tf32x3"])
        ctx.set_stream(torch.cuda.current_stream().cuda_stream)
        ctx.set_spins(asd.random_spins(N, nf, seed=0), as_origin=True)
        d = torch.zeros(2, dtype=torch.float64, device="cuda")
        ctx.step(3)
        step_ms = timed(torch, lambda: (ctx.step(1), ctx.sqt_async("bf16x3", d.data_ptr())),
                        args.steps)
        llg_ms = {}
        for kern in ("stages", "fused"):
            ctx.set_llg_kernel(kern)
            ctx.step(2)
            llg_ms[kern] = timed(torch, lambda: ctx.step(1), 10)
        ctx.set_llg_kernel("auto")
        vals, ms = {}, {}
        for mode, reps in (("bf16x3", 5), ("tf32x3", 3), ("fp64", 1)):
            ctx.sqt_async(mode, d.data_ptr())
            ms[mode] = timed(torch, lambda: ctx.sqt_async(mode, d.data_ptr()), reps)
            vals[mode] = complex(*d.tolist())
        flops = 2.0 * M * M * K
        out.update({
            "metric": METRIC, "value": M * nf / (step_ms / 1e3), "unit": "site-steps/s",
            "ms_per_step": step_ms, "dtype": "f64 RK4 + bf16x3 GEMM",
            "config": {"workload": "256x256 lattice, 1000 replicas, J=1, J2=-0.3, alpha=0.02, dt=0.005",
                       "gemm_m": M, "gemm_k": K},
            "llg": llg_report(llg_ms, M * nf, llg_fp64_ops(True, False, True), hbm,
                              fp64_peak_tops(torch)),
            "sqt": {m: {"ms": ms[m], "tflops": flops / ms[m] / 1e9,
                        "rel_err_vs_fp64": abs(vals[m] - vals["fp64"]) / abs(vals["fp64"])}
                    for m in ms},
            "sqt_speedup_vs_fp64": {m: ms["fp64"] / ms[m] for m in ("bf16x3", "tf32x3")},
            "roofline": {"bound": "tensor", "kernel": "umma_sqt_kernel (bf16x3)",
                         "achieved": flops / ms["bf16x3"] / 1e9, "peak": bf16, "unit": "TFLOP/s",
                         "frac": flops / ms["bf16x3"] / 1e9 / bf16, "traffic": None,
                         **split_ceiling("bf16x3", flops / ms["bf16x3"] / 1e9 / bf16)},
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
    """--shard: the headline ensemble (128x128, 500 replicas) split by replicas
    over the ranks -- strong scaling of one system.  Each rank steps its
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
    N, nf = CONFIG["N"], CONFIG["nfile"]
    M = N * N
    b, e = shard_range(nf, rank, world)
    mode = args.mode
    params = asd.Params.make(N, e - b, J1=CONFIG["J1"], J2=CONFIG["J2"], alpha=CONFIG["alpha"],
                             h=CONFIG["h"], dt=CONFIG["dt"])
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
        "config": {"workload": WORKLOAD + ", one ensemble split by replicas", "sites": M,
                   "replicas": nf, "parallelism": f"replicas/{world}", "sqt_mode": mode,
                   "exchange_doubles_per_step": 2 + 3 * M,
                   "l2": "inputs larger than L2 at 1 and 2 GPUs"},
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
    ap.add_argument("--mode", choices=["tf32x3", "bf16x3", "fp64", "fp64_fused"], default="tf32x3")
    ap.add_argument("--batch-cluster", type=int, default=0,
                    help="batch48: clusters of this many CTAs instead of the autotuner's choice")
    ap.add_argument("--llg-kernel", choices=["auto", "fused", "stages"], default="auto",
                    help="RK4 step of the headline: one streamed launch where it fills the GPU "
                         "(auto, default), always (fused) or four stage kernels (stages)")
    ap.add_argument("--chunk-k", type=int, default=-1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="only the timed steps (for profiling): no per-component timings, e2e "
                         "or CPU baseline after the timed region")
    ap.add_argument("--ref-target-s", type=float, default=2.0)
    ap.add_argument("--workload", choices=["headline", "grid32", "sqt256", "adjoint64", "batch48"],
                    default="headline", help="secondary workloads print their own line")
    ap.add_argument("--shard", action="store_true",
                    help="strong scaling: split the one headline ensemble by replicas over the "
                         "ranks (S(q,t) exchanged every step) instead of one ensemble per rank")
    args = ap.parse_args()
    if args.workload != "headline":
        return run_workload(args)
    if args.shard and args.impl == "ours":
        return run_sharded(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
