"""GPU parity of the LLG time stepping (through the C ABI) against the oracle.

The stage kernels use explicitly rounded FP64 operations in the reference's
order, so the comparison is bit for bit: the tolerance is zero."""
from __future__ import annotations

import numpy as np
import pytest

import asd_b200 as asd
import oracle as orc

pytestmark = pytest.mark.gpu

CASES = [
    # N, nfile, kwargs
    (12, 4, dict(J1=1.0, dt=0.02)),
    (20, 6, dict(J1=-1.0, dt=0.01)),
    (9, 33, dict(J1=0.7, dt=0.03)),                      # odd N, ragged replica count
    (16, 3, dict(J1=1.0, dt=0.01, spin_len=1.5)),        # the fusion program's length
    (24, 5, dict(J1=-1.0, alpha=0.05, h=(0.0, 0.0, 0.5), dt=0.005)),
    (16, 7, dict(J1=1.0, J2=-0.3, alpha=0.02, dt=0.005)),
    (10, 2, dict(J1=1.0, alpha=0.1, dt=0.01)),
    (3, 1, dict(J1=1.0, J2=0.5, h=(0.1, 0.2, 0.3), alpha=0.3, dt=0.02)),   # smallest lattice
    (37, 9, dict(J1=-0.8, J2=0.2, h=(0.0, 0.3, 0.1), alpha=0.07, dt=0.01)),  # ragged tiles
    (48, 4, dict(J1=1.0, dt=0.02)),                      # several whole tiles
    # more combinations of the extensions, even and odd replica counts
    (14, 8, dict(J1=-1.0, J2=0.3, alpha=0.05, h=(0.1, 0.0, 0.4), dt=0.005)),
    (11, 6, dict(J1=0.9, J2=-0.2, h=(0.0, 0.2, 0.0), dt=0.01)),
    (7, 2, dict(J1=1.0, h=(0.0, 0.0, 0.5), alpha=0.2, dt=0.02, spin_len=1.5)),
    # column bands of the one-launch step: 2 bands of 40, 3 of 48 (the last
    # ragged), 4 of 64; replica groups of 4 with a partial last group
    (70, 13, dict(J1=1.0, J2=-0.3, alpha=0.02, dt=0.005)),
    (130, 5, dict(J1=-1.0, alpha=0.05, h=(0.0, 0.0, 0.5), dt=0.005)),
    (256, 3, dict(J1=1.0, J2=-0.3, h=(0.2, 0.0, 0.1), alpha=0.02, dt=0.005)),
    # 64 or more replicas: the stage kernels' blocks of 2 x 4 sites x 32
    # replicas.  Odd replica count with a last group of 1 and ragged blocks;
    # with and without J2; N = 3, narrower than one block, so neighbours wrap
    # onto the block's own sites; a last group of 6 with every extension;
    # N = 70, ragged in both directions, with a last group of 2.
    (9, 65, dict(J1=0.7, J2=0.4, dt=0.03)),
    (6, 96, dict(J1=-1.0, alpha=0.05, h=(0.0, 0.0, 0.5), dt=0.005)),
    (3, 64, dict(J1=1.0, J2=-0.3, alpha=0.1, dt=0.01)),
    (13, 70, dict(J1=1.0, J2=-0.3, h=(0.1, 0.2, 0.0), alpha=0.02, dt=0.005, spin_len=1.5)),
    (5, 67, dict(J1=1.0, dt=0.02)),
    (70, 66, dict(J1=-1.0, J2=0.2, alpha=0.05, dt=0.005)),
]


@pytest.mark.parametrize("kernel", ["fused", "stages", "auto"])
@pytest.mark.parametrize("N,nfile,kw", CASES)
def test_ctx_steps_bit_exact(oracle, N, nfile, kw, kernel):
    s0 = asd.random_spins(N, nfile, seed=N + nfile, spin_len=kw.get("spin_len", 1.0))
    with asd.Context(asd.Params.make(N, nfile, **kw), modes=["fp64"]) as ctx:
        ctx.set_llg_kernel(kernel)
        ctx.set_spins(s0, as_origin=True)
        assert np.array_equal(ctx.get_spins(), s0)  # layout round trip
        ctx.step(5)
        got = ctx.get_spins()
    want = oracle.steps(orc.make_params(N, nfile, **kw), s0, 5)
    assert np.array_equal(got, want), np.abs(got - want).max()


@pytest.mark.parametrize("kernel", ["fused", "stages"])
@pytest.mark.parametrize("name", ["llg_n12_f4", "llg_n20_f6"])
def test_ctx_matches_reference_fixture(golden, name, kernel):
    g = golden(name)
    N, nf, n = int(g["N"]), int(g["nfile"]), int(g["nsteps"])
    for length, key in ((1.0, "steps_len1"), (1.5, "steps_len15")):
        p = asd.Params.make(N, nf, J1=float(g["J1"]), dt=float(g["dt"]), spin_len=length)
        with asd.Context(p, modes=["fp64"]) as ctx:
            ctx.set_llg_kernel(kernel)
            ctx.set_spins(g["spins0"], as_origin=True)
            ctx.step(n)
            assert np.array_equal(ctx.get_spins(), g[key])


def test_dropin_euler_and_runge_kutta_bit_exact(golden):
    g = golden("llg_n12_f4")
    asd.set_params(int(g["N"]), int(g["nfile"]), float(g["J1"]), float(g["dt"]))
    assert np.array_equal(asd.euler(g["spins0"]), g["euler"])
    cur, k1, k2, k3, k4 = asd.runge_kutta(g["spins0"])
    for mine, key in zip((cur, k1, k2, k3, k4), ("rk_cur", "rk_k1", "rk_k2", "rk_k3", "rk_k4")):
        assert np.array_equal(mine, g[key]), key


def test_dropin_random_sizes(oracle):
    for N, nf in ((5, 1), (31, 3), (64, 2)):
        s = asd.random_spins(N, nf, seed=N)
        asd.set_params(N, nf, 1.0, 0.02)
        p = orc.make_params(N, nf, J1=1.0, dt=0.02)
        assert np.array_equal(asd.euler(s), oracle.deriv(p, s))
        got = asd.runge_kutta(s)
        want = oracle.rk4(p, s)
        for a, b in zip(got, want):
            assert np.array_equal(a, b)


def test_long_run_stays_on_sphere():
    N, nf = 32, 8
    s0 = asd.random_spins(N, nf, seed=1)
    with asd.Context(asd.Params.make(N, nf, J1=-1.0, alpha=0.05, h=(0, 0, 0.5), dt=0.005)) as ctx:
        ctx.set_spins(s0, as_origin=True)
        ctx.step(200)
        out = ctx.get_spins()
    assert np.allclose(np.linalg.norm(out, axis=-1), 1.0, atol=1e-15)


def test_constant_division_is_correctly_rounded():
    """The stage kernels divide by 3 and 6 with Markstein's correction step;
    it must equal the correctly rounded division bit for bit over the range
    the RK4 increments use and well beyond it."""
    import torch

    g = torch.Generator(device="cuda").manual_seed(5)
    n = 1 << 24
    mant = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) + 1.0
    expo = torch.randint(-300, 300, (n,), device="cuda", generator=g).double()
    sign = torch.where(torch.rand(n, device="cuda", generator=g) < 0.5, -1.0, 1.0).double()
    x = (sign * mant * torch.exp2(expo)).contiguous()
    # plus dense samples around typical increments and exact multiples of 3
    y = (torch.rand(n, dtype=torch.float64, device="cuda", generator=g) - 0.5) * 0.1
    z = torch.arange(-(1 << 20), 1 << 20, dtype=torch.float64, device="cuda") * 3.0 * 2.0 ** -30
    special = torch.tensor([0.0, -0.0, 1.0, -1.0, 3.0, 6.0, 1e-300, -1e-300, 2.0 ** -1000],
                           dtype=torch.float64, device="cuda")
    bad = torch.zeros(1, dtype=torch.int64, device="cuda")
    for arr in (x, y, z, special):
        asd.check_const_division(arr.data_ptr(), arr.numel(), bad.data_ptr(),
                                 torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(bad.item()) == 0
