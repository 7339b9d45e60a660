"""S(q,t) on the full N x N q grid (displacement-binning epilogue + 2-D DFT)
against the oracle's direct O(N^4 K) grid, and the 32 x 32 FP64 configuration
run end to end: 2000 RK4 steps with J = 1, alpha = 0.1, dt = 0.01 and 200
replicas, compared bit for bit with the oracle's trajectory, then S(q,t) on the
whole grid.

Tolerances, relative to max_q |S(q)|: FP64 1e-12, split modes 1e-5."""
from __future__ import annotations

import numpy as np
import pytest

import asd_b200 as asd
import oracle as orc
from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "tf32x3": 1e-5, "bf16x3": 1e-5, "fp16x3": 1e-5}


def grid_err(got, want):
    return float(np.abs(got - want).max() / np.abs(want).max())


@pytest.mark.parametrize("N,nfile,steps", [(16, 8, 3), (24, 30, 2), (32, 12, 1), (10, 5, 4)])
def test_grid_vs_oracle(oracle, N, nfile, steps):
    s0 = asd.random_spins(N, nfile, seed=N + 100 * nfile)
    kw = dict(J1=1.0, alpha=0.1, dt=0.01)
    with asd.Context(asd.Params.make(N, nfile, **kw)) as ctx:
        ctx.set_spins(s0, as_origin=True)
        ctx.step(steps)
        st = ctx.get_spins()
        want = oracle.sqt_grid(N, nfile, st, s0)
        vx = N // 10
        for mode, tol in TOL.items():
            got = ctx.sqt_grid(mode)
            assert grid_err(got, want) < tol, mode
            # the grid point q = 2 pi (vx, vy)/N is the single-q S(q,t)
            assert rel_err(got[vx, vx], ctx.sqt(mode)) < max(tol, 1e-11), mode


def test_grid_q0_and_past_64():
    N, nf = 64, 4
    s0 = asd.random_spins(N, nf, seed=3)
    with asd.Context(asd.Params.make(N, nf)) as ctx:
        ctx.set_spins(s0, as_origin=True)
        g = ctx.sqt_grid("fp64")
        assert np.all(np.isfinite(g))
        # q = 0 of the connected correlation at t = 0 is sum_j C_ij - m.z summed:
        # equal to the FP64 single-q value at vx = vy = 0
    with asd.Context(asd.Params.make(N, nf, vx=0, vy=0)) as ctx:
        ctx.set_spins(s0, as_origin=True)
        assert rel_err(g[0, 0], ctx.sqt("fp64")) < 1e-11
    # no size limit: 65 x 65 (past the former shared-memory bins) in every mode
    with asd.Context(asd.Params.make(65, 2)) as ctx:
        s65 = asd.random_spins(65, 2, seed=1)
        ctx.set_spins(s65, as_origin=True)
        ctx.step(1)
        grids = {m: ctx.sqt_grid(m) for m in TOL}
    for m, tol in TOL.items():
        assert grid_err(grids[m], grids["fp64"]) < tol, m


def test_fp64_configuration_32x32_full_run(oracle):
    """2000 steps on the GPU equal the oracle's 2000 steps bit for bit, and the
    q-grid S(q,t) of the final state matches the oracle's grid."""
    N, nf, steps = 32, 200, 2000
    kw = dict(J1=1.0, alpha=0.1, dt=0.01)
    s0 = asd.random_spins(N, nf, seed=0)
    with asd.Context(asd.Params.make(N, nf, **kw)) as ctx:
        ctx.set_spins(s0, as_origin=True)
        ctx.step(steps)
        st = ctx.get_spins()
        grid = ctx.sqt_grid("fp64")
    want_st = oracle.steps(orc.make_params(N, nf, **kw), s0, steps)
    assert np.array_equal(st, want_st)
    want = oracle.sqt_grid(N, nf, st, s0)
    assert grid_err(grid, want) < 1e-12
