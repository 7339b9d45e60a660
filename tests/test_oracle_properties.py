"""Properties of the LLG flow and of S(q,t) that hold for any correct
implementation (used to pin the extensions the reference does not have:
damping, Zeeman field, next-nearest exchange)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as orc
from conftest import rel_err


def test_uniform_ferromagnet_is_stationary(oracle):
    N, nf = 8, 3
    s = np.zeros((nf, N * N, 3))
    s[..., 2] = 1.0
    p = orc.make_params(N, nf, J1=1.3, J2=-0.4, alpha=0.1, dt=0.01)
    assert np.all(oracle.deriv(p, s) == 0.0)
    assert np.array_equal(oracle.steps(p, s, 5), s)


@pytest.mark.parametrize("spin_len", [1.0, 1.5])
def test_renormalisation_keeps_length(oracle, spin_len):
    N, nf = 10, 4
    s = orc.random_spins(N, nf, seed=1, spin_len=spin_len)
    p = orc.make_params(N, nf, J1=-1.0, J2=0.3, alpha=0.05, h=(0.1, 0.0, 0.5), dt=0.02,
                        spin_len=spin_len)
    out = oracle.steps(p, s, 7)
    assert np.allclose(np.linalg.norm(out, axis=-1), spin_len, rtol=0, atol=4e-16 * spin_len * 4)


def test_extensions_reduce_to_reference(oracle):
    """alpha = J2 = h = 0 must be the reference's equation; with them on, the
    derivative equals the closed form -g [S x H + alpha S x (S x H)]."""
    N, nf = 7, 2
    s = orc.random_spins(N, nf, seed=4)
    p0 = orc.make_params(N, nf, J1=0.9)
    p = orc.make_params(N, nf, J1=0.9, J2=-0.3, alpha=0.2, h=(0.1, -0.2, 0.3))
    d = oracle.deriv(p, s)
    S = s.reshape(nf, N, N, 3)
    H = 0.9 * (np.roll(S, -1, 1) + np.roll(S, 1, 1) + np.roll(S, 1, 2) + np.roll(S, -1, 2))
    H += -0.3 * (np.roll(S, (-1, -1), (1, 2)) + np.roll(S, (-1, 1), (1, 2)) +
                 np.roll(S, (1, -1), (1, 2)) + np.roll(S, (1, 1), (1, 2)))
    H += np.array([0.1, -0.2, 0.3])
    sxh = np.cross(S, H)
    expect = -(sxh + 0.2 * np.cross(S, sxh)) / (1 + 0.2 ** 2)
    assert np.allclose(d.reshape(expect.shape), expect, atol=1e-14)
    d0 = oracle.deriv(p0, s).reshape(nf, N, N, 3)
    H0 = 0.9 * (np.roll(S, -1, 1) + np.roll(S, 1, 1) + np.roll(S, 1, 2) + np.roll(S, -1, 2))
    assert np.allclose(d0, np.cross(H0, S), atol=1e-15)


def test_damping_relaxes_towards_field(oracle):
    N, nf = 4, 2
    s = orc.random_spins(N, nf, seed=9)
    p = orc.make_params(N, nf, J1=0.0, alpha=0.5, h=(0.0, 0.0, 1.0), dt=0.05)
    out = oracle.steps(p, s, 400)
    assert np.all(out[..., 2] > 0.999)


def test_sqt_connected_part_vanishes_for_identical_replicas(oracle):
    """With all replicas equal, C_ij equals the outer product of the means and
    the connected S(q,t) is zero; the baseline's non-connected form is not."""
    N, nf = 12, 3
    one = orc.random_spins(N, 1, seed=5)
    s = np.repeat(one, nf, axis=0)
    vx = N // 10
    assert abs(oracle.sqt_gemm(N, nf, vx, vx, s, s)) < 1e-13
    assert abs(oracle.sqt_factorized(N, nf, vx, vx, s, s)) < 1e-13
    assert abs(oracle.sqt_direct(N, nf, vx, vx, s, s)) > 1e-3


def test_sqt_forms_agree(oracle):
    N, nf = 16, 5
    s0 = orc.random_spins(N, nf, seed=6)
    p = orc.make_params(N, nf, J1=1.0, dt=0.02)
    st = oracle.steps(p, s0, 3)
    vx = N // 10
    ref = oracle.sqt_gemm(N, nf, vx, vx, st, s0)
    assert rel_err(oracle.sqt_fused(N, nf, vx, vx, st, s0), ref) < 1e-13
    assert rel_err(oracle.sqt_factorized(N, nf, vx, vx, st, s0), ref) < 1e-13
    grid = oracle.sqt_grid(N, nf, st, s0)
    assert rel_err(grid[vx, vx], ref) < 1e-13
    # q and -q are complex conjugates for real spins
    assert abs(grid[vx, vx] - np.conj(grid[(-vx) % N, (-vx) % N])) < 1e-12


def _energy(s, N, J1, J2, h):
    """E = -J1 sum_bonds S_i.S_j - J2 sum_diagonal_bonds S_i.S_j - h.sum S_i per
    replica, each bond once, so that -dE/dS_i is the effective field the
    derivative uses (J1 over the 4 nearest, J2 over the 4 diagonal
    neighbours, plus h)."""
    S = s.reshape(s.shape[0], N, N, 3)
    nn = (S * np.roll(S, -1, 1)).sum((1, 2, 3)) + (S * np.roll(S, -1, 2)).sum((1, 2, 3))
    nnn = ((S * np.roll(S, (-1, -1), (1, 2))).sum((1, 2, 3)) +
           (S * np.roll(S, (-1, 1), (1, 2))).sum((1, 2, 3)))
    return -J1 * nn - J2 * nnn - (S * np.asarray(h)).sum((1, 2, 3))


def test_energy_is_conserved_to_fourth_order_without_damping(oracle):
    """Precession conserves E exactly, so its drift over a fixed time is RK4's
    global error: it must shrink about 2^4 = 16-fold per halving of dt."""
    N, nf = 12, 3
    kw = dict(J1=1.0, J2=-0.3, h=(0.1, 0.0, 0.5))
    s0 = orc.random_spins(N, nf, seed=5)
    E0 = _energy(s0, N, **kw)
    drift = []
    for dt, n in ((0.02, 50), (0.01, 100), (0.005, 200)):  # to t = 1 each
        s = oracle.steps(orc.make_params(N, nf, alpha=0.0, dt=dt, **kw), s0, n)
        drift.append(np.abs(_energy(s, N, **kw) - E0).max() / np.abs(E0).max())
    assert drift[1] < 1e-7
    assert drift[0] / drift[1] > 12 and drift[1] / drift[2] > 12, drift


def test_damping_dissipates_energy_every_step(oracle):
    """With Gilbert damping dE/dt = -g alpha sum |H x S|^2 <= 0: E falls at
    every step (J2 and the field included)."""
    N, nf = 12, 3
    kw = dict(J1=1.0, J2=-0.3, h=(0.1, 0.0, 0.5))
    p = orc.make_params(N, nf, alpha=0.1, dt=0.01, **kw)
    s = orc.random_spins(N, nf, seed=6)
    E = [_energy(s, N, **kw)]
    for _ in range(100):
        s = oracle.steps(p, s, 1)
        E.append(_energy(s, N, **kw))
    assert np.all(np.diff(np.array(E), axis=0) < 0)
