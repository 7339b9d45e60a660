"""The C programs on the GPU: the driver (host/llg_sqt, context API) and a
program written like the reference's kernel-fusion driver that uses the
drop-in euler/runge_kutta/fused_dgemm through the reference's own globals.
Both are compared with the oracle: spins bit for bit, S(q,t) to 1e-12."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

import asd_b200 as asd
import oracle as orc
from conftest import PKG, ROOT, rel_err

pytestmark = pytest.mark.gpu


def parse(stdout, tag):
    vals = {}
    for line in stdout.splitlines():
        f = line.split()
        if f and f[0] == tag:
            key = tuple(int(x) for x in f[1:-2])
            vals[key] = complex(float(f[-2]), float(f[-1]))
    return vals


def test_driver_program(oracle, tmp_path):
    subprocess.run(["make", "-C", str(PKG), "host/llg_sqt"], check=True, capture_output=True)
    N, nf, steps = 20, 6, 7
    s0 = asd.random_spins(N, nf, seed=9)
    src, dst = tmp_path / "in.spins", tmp_path / "out.spins"
    asd.save_spins(src, s0)
    r = subprocess.run([str(PKG / "host" / "llg_sqt"), "-i", str(src), "-o", str(dst), "-m",
                        str(steps), "-w", "2", "-e", "0.01", "-J", "-1", "-a", "0.05", "-H",
                        "0,0,0.5", "-q", "fp64", "-p", "-g", "-r", str(tmp_path / "t.txt")],
                       capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    p = orc.make_params(N, nf, J1=-1.0, alpha=0.05, h=(0, 0, 0.5), dt=0.01)
    got, step, _ = asd.load_spins(dst)
    assert step == steps
    assert np.array_equal(got, oracle.steps(p, s0, steps))
    sqt = parse(r.stdout, "sqt")
    assert len(sqt) == steps
    st = s0
    for k in range(steps):
        st = oracle.steps(p, st, 1)
        assert rel_err(sqt[(k,)], oracle.sqt_factorized(N, nf, 2, 2, st, s0)) < 1e-12
    grid = parse(r.stdout, "sqt_grid")
    want = oracle.sqt_grid(N, nf, st, s0)
    got_g = np.array([[grid[(a, b)] for b in range(N)] for a in range(N)])
    assert np.abs(got_g - want).max() < 1e-12 * np.abs(want).max()
    line = (tmp_path / "t.txt").read_text().split()
    assert int(line[0]) == N and float(line[1]) > 0 and float(line[2]) > 0


def test_reference_style_program_uses_dropin_symbols(oracle, tmp_path):
    exe = tmp_path / "dropin_host"
    subprocess.run(["gcc", "-O2", "-o", str(exe), str(ROOT / "tests" / "dropin_host.c"),
                    f"-I{ROOT / 'include'}", f"-L{PKG / 'lib'}", "-lasd_b200",
                    f"-Wl,-rpath,{PKG / 'lib'}", "-lm"], check=True)
    N, nf, steps, dt, J1 = 12, 4, 3, 0.02, 1.0
    s0 = asd.random_spins(N, nf, seed=21)
    src, dst = tmp_path / "in.spins", tmp_path / "out.spins"
    asd.save_spins(src, s0)
    r = subprocess.run([str(exe), str(src), str(dst), str(steps), str(dt), str(J1)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    p = orc.make_params(N, nf, J1=J1, dt=dt)
    got, _, _ = asd.load_spins(dst)
    assert np.array_equal(got, oracle.steps(p, s0, steps))
    sqt = parse(r.stdout, "sqt")
    st = s0
    for k in range(steps):
        st = oracle.steps(p, st, 1)
        assert rel_err(sqt[(k,)], oracle.sqt_fused(N, nf, N // 10, N // 10, st, s0)) < 1e-12
