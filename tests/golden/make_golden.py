"""Generates tests/golden/*.npz from the reference's OWN compiled functions.

Run in a container that has the reference sources (the build compiles them
into oracle/_ref/ with ``make -C oracle ref``):

    python tests/golden/make_golden.py

Every fixture stores its inputs too, so the tests never regenerate random
numbers.  The reference ships no test vectors of its own; these come from its
euler / runge_kutta (llg_sqt_baseline.c:29-142), its renormalisation loop
(llg_sqt_baseline.c:298-309, llg_sqt_fusion.c:350-361), its fused_dgemm
(kernel_fusion/gemm_kernel.h:355-422) and its OpenBLAS S(q,t) sequence
(gemm/llg_sqt_mkl.c:349-423), driven by oracle/ref_glue.c.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
from oracle import RefLib, build, random_spins  # noqa: E402

OUT = Path(__file__).resolve().parent


def llg_case(name, N, nfile, J1, dt, seed, nsteps, full=True):
    spins0 = random_spins(N, nfile, seed)
    fx = {"N": N, "nfile": nfile, "J1": J1, "dt": dt, "nsteps": nsteps, "spins0": spins0}
    for variant in ("baseline", "fusion", "gemm"):
        r = RefLib(variant)
        r.setup(N, nfile, J1=J1, dt=dt, threads=4)
        fx["vx"] = r.lib.ref_get_vx()
        if variant == "baseline":
            if full:
                fx["euler"] = r.euler(spins0)
                cur, k1, k2, k3, k4 = r.runge_kutta(spins0)
                fx.update(rk_cur=cur, rk_k1=k1, rk_k2=k2, rk_k3=k3, rk_k4=k4)
            fx["steps_len1"] = r.steps(spins0, nsteps, 1.0)
        elif variant == "fusion":
            fx["steps_len15"] = r.steps(spins0, nsteps, 1.5)
            r.fusion_init(spins0)
            fx["sqt_fused_len1"] = np.array(r.fusion_sqt(fx["steps_len1"]))
        else:
            fx["sqt_gemm_len1"] = np.array(r.gemm_sqt(fx["steps_len1"], spins0))
    np.savez_compressed(OUT / f"{name}.npz", **fx)
    print(name, "S(q,t) fused", fx["sqt_fused_len1"], "gemm", fx["sqt_gemm_len1"])


def fused_dgemm_case(name, m, n, k, seed):
    rng = np.random.default_rng(seed)
    lda, ldb = m + 3, k + 2
    ldc = 2 * ((m + 3) // 4) * 4 + 8
    a = rng.standard_normal(lda * k)
    b = rng.standard_normal(ldb * n)
    c = rng.standard_normal(ldc * n)
    q = rng.standard_normal(ldc * n)
    alpha = 1.0 / 7.0
    r = RefLib("fusion")
    r.setup(8, 1, threads=4)
    c_out = c.copy()
    sum_ = np.zeros(2 * 128)
    r.lib.ref_fused_dgemm(m, n, k, alpha, a, lda, b, ldb, c_out, ldc, q, sum_)
    total = np.array([sum_[0::2].sum(), sum_[1::2].sum()])
    np.savez_compressed(OUT / f"{name}.npz", m=m, n=n, k=k, lda=lda, ldb=ldb, ldc=ldc, a=a, b=b,
                        c_in=c, q=q, alpha=alpha, c_out=c_out, sum=total)
    print(name, "sum", total)


def main():
    build(quiet=False)
    llg_case("llg_n12_f4", N=12, nfile=4, J1=1.0, dt=0.02, seed=11, nsteps=10)
    llg_case("llg_n20_f6", N=20, nfile=6, J1=-1.0, dt=0.01, seed=12, nsteps=6, full=False)
    fused_dgemm_case("fused_dgemm_valid", m=32, n=12, k=96, seed=21)
    # each edge on its own: rows past the last multiple of 4 with K > 240, and
    # an odd last column with K > 240.  (Both together are not a fixture: the
    # reference's result then depends on its thread count, gemm_kernel.h:206.)
    fused_dgemm_case("fused_dgemm_rows", m=34, n=12, k=300, seed=22)
    fused_dgemm_case("fused_dgemm_cols", m=32, n=7, k=300, seed=23)


if __name__ == "__main__":
    main()
