"""bench.py's output contract, on the CPU: the reference arm (the reference's
own programs on the host cores) prints one JSON line with the keys the
driver reads and the same `config` as the GPU arm; ranks other than 0 exit
without work; the whole-job aggregation takes the slowest rank."""
from __future__ import annotations

import json
import os
import subprocess
import sys
import types
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _bench():
    sys.path.insert(0, str(ROOT))
    import bench

    return bench


def _run(*extra, env=None):
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", *extra]
    e = dict(os.environ, **(env or {}))
    p = subprocess.run(cmd, cwd=ROOT, env=e, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    return [json.loads(l) for l in p.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_line():
    lines = _run("--steps", "1", "--warmup", "0", "--ref-target-s", "0.02")
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference"
    if "unavailable" in d:  # the reference was not compiled in this checkout
        assert isinstance(d["unavailable"], str) and d["unavailable"]
        pytest.skip(d["unavailable"])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["unit"] == "site-steps/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "site-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    # the same workload description as the GPU arm, key for key
    bench = _bench()
    args = types.SimpleNamespace(mode=None, llg_kernel="auto", chunk_k=-1)
    assert d["config"] == bench.bench_config("sqt256", args)
    # the fused program's S(q,t) is invalid at K = 3000 > 240: timed, labelled
    fused = d["paths"]["fused_avx2"]
    assert fused["value_valid"] is False and fused["value"] > 0


def test_reference_arm_other_ranks_do_no_work():
    lines = _run("--steps", "1", "--warmup", "0",
                 env={"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert lines == []


def test_aggregate_takes_the_slowest_rank():
    bench = _bench()
    ms, value = bench.aggregate(50.0, 1e6, 1)
    assert ms == 50.0 and value == pytest.approx(2e7)
    # weak scaling: every rank did units_per_rank in its own time
    ms, value = bench.aggregate(50.0, 1e6, 4)
    assert value == pytest.approx(8e7)


def test_llg_fraction_per_clock():
    """The FP64 fraction at equal clocks scales the sustained fraction by the
    FMA kernel's clock over the LLG kernel's; without both clocks it is not
    reported."""
    bench = _bench()
    llg = bench.llg_report({"fused": 4.0}, 6.5536e7, 387, 6538.0, 16.9, 16.9)
    frac = llg["fused"]["fp64_frac_sustained"]
    bench.add_per_clock(llg, {"fused": {"sm_mhz": 1500}}, {"sm_mhz": 1965})
    assert llg["fused"]["fp64_frac_per_clock"] == pytest.approx(frac * 1965 / 1500)
    llg2 = bench.llg_report({"fused": 4.0}, 6.5536e7, 387, 6538.0, 16.9, 16.9)
    bench.add_per_clock(llg2, None, {"sm_mhz": 1965})
    assert "fp64_frac_per_clock" not in llg2["fused"]


@pytest.mark.parametrize("name,mode,label", [("sqt256", None, "BF16x3"), ("sqt128", None, "TF32x3"),
                                             ("sqt128", "bf16x3", "BF16x3"),
                                             ("sqt256", "fp16x3", "FP16x3")])
def test_config_names_the_mode_it_runs(name, mode, label):
    """The workload string and sqt_mode name the S(q,t) mode a run uses,
    also when --mode overrides the workload's own."""
    bench = _bench()
    args = types.SimpleNamespace(mode=mode, llg_kernel="auto", chunk_k=-1)
    cfg = bench.bench_config(name, args)
    assert cfg["workload"].endswith(f"S(q,t) in {label}")
    assert cfg["sqt_mode"] == label.lower()
    assert cfg["chunk_k"] == (512 if label == "TF32x3" else 1024)
