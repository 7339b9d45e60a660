"""Pins the CPU oracle (oracle/asd_oracle.c) to the reference.

* against the golden fixtures, which the reference's own compiled functions
  produced (tests/golden/make_golden.py);
* against the live reference libraries (oracle/_ref/), when they were built.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as orc
from conftest import rel_err

LLG_CASES = ["llg_n12_f4", "llg_n20_f6"]
DGEMM_CASES = ["fused_dgemm_valid", "fused_dgemm_rows", "fused_dgemm_cols"]


@pytest.mark.parametrize("name", LLG_CASES)
def test_oracle_trajectory_matches_reference_bit_exact(oracle, golden, name):
    g = golden(name)
    N, nf = int(g["N"]), int(g["nfile"])
    p = orc.make_params(N, nf, J1=float(g["J1"]), dt=float(g["dt"]))
    if "euler" in g:
        assert np.array_equal(oracle.deriv(p, g["spins0"]), g["euler"])
        cur, k1, k2, k3, k4 = oracle.rk4(p, g["spins0"])
        for mine, key in zip((cur, k1, k2, k3, k4), ("rk_cur", "rk_k1", "rk_k2", "rk_k3", "rk_k4")):
            assert np.array_equal(mine, g[key]), key
    assert np.array_equal(oracle.steps(p, g["spins0"], int(g["nsteps"])), g["steps_len1"])
    p.spin_len = 1.5
    assert np.array_equal(oracle.steps(p, g["spins0"], int(g["nsteps"])), g["steps_len15"])


@pytest.mark.parametrize("name", LLG_CASES)
def test_oracle_sqt_matches_reference(oracle, golden, name):
    g = golden(name)
    N, nf, vx = int(g["N"]), int(g["nfile"]), int(g["vx"])
    st, s0 = g["steps_len1"], g["spins0"]
    ref_fused = complex(g["sqt_fused_len1"])
    ref_gemm = complex(g["sqt_gemm_len1"])
    assert rel_err(ref_fused, ref_gemm) < 1e-13  # the reference agrees with itself
    for fn in (oracle.sqt_fused, oracle.sqt_gemm, oracle.sqt_factorized):
        assert rel_err(fn(N, nf, vx, vx, st, s0), ref_fused) < 1e-13, fn.__name__
    grid = oracle.sqt_grid(N, nf, st, s0)
    assert rel_err(grid[vx, vx], ref_gemm) < 1e-13


@pytest.mark.parametrize("name", DGEMM_CASES)
def test_oracle_fused_dgemm_matches_reference(oracle, golden, name):
    g = golden(name)
    c = g["c_in"].copy()
    s = np.zeros(2)
    oracle.fused_dgemm(int(g["m"]), int(g["n"]), int(g["k"]), float(g["alpha"]), g["a"],
                       int(g["lda"]), g["b"], int(g["ldb"]), c, int(g["ldc"]), g["q"], s)
    assert np.array_equal(c, g["c_out"])  # same FMA chain per element
    assert np.allclose(s, g["sum"], rtol=1e-13, atol=1e-12)


@pytest.mark.skipif(not orc.RefLib.available("baseline"), reason="reference libraries not built")
@pytest.mark.parametrize("N,nfile,J1,dt", [(6, 3, 1.0, 0.02), (13, 5, -0.7, 0.013), (32, 2, 1.0, 0.05)])
def test_oracle_vs_live_reference(oracle, N, nfile, J1, dt):
    spins = orc.random_spins(N, nfile, seed=N * 7 + nfile)
    r = orc.RefLib("baseline")
    r.setup(N, nfile, J1=J1, dt=dt, threads=2)
    p = orc.make_params(N, nfile, J1=J1, dt=dt)
    assert np.array_equal(r.euler(spins), oracle.deriv(p, spins))
    assert np.array_equal(r.steps(spins, 4, 1.0), oracle.steps(p, spins, 4))


@pytest.mark.skipif(not orc.RefLib.available("fusion"), reason="reference libraries not built")
def test_oracle_sqt_vs_live_reference_fused(oracle):
    N, nf = 20, 8
    s0 = orc.random_spins(N, nf, seed=3)
    p = orc.make_params(N, nf, J1=1.0, dt=0.02)
    st = oracle.steps(p, s0, 3)
    r = orc.RefLib("fusion")
    r.setup(N, nf, threads=4)
    r.fusion_init(s0)
    vx = N // 10
    assert rel_err(r.fusion_sqt(st), oracle.sqt_fused(N, nf, vx, vx, st, s0)) < 1e-13
