"""Gradients of the S(q,t)-mismatch loss (asd_ctx_loss_grad, the adjoint RK4
with checkpointed recomputation) against

* an FP64 reference gradient: torch autograd through a plain torch FP64
  implementation of the same forward (RK4, renormalisation, S(q,t));
* central finite differences on the differentiation configuration: 64 x 64
  lattice, 100 replicas, 1000 steps, S(q,t) every 10 steps, checkpoints every
  50 steps, target from J = 1, alpha = 0.1, h = (0, 0, 0.2), gradient at
  J = 0.8, alpha = 0.15, h = 0 -- tolerance 1e-4 relative.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import asd_b200 as asd

pytestmark = pytest.mark.gpu


def torch_loss(theta, s0, N, nf, dt, nsteps, stride, vx, target, spin_len=1.0):
    import torch

    J1, J2, al, hx, hy, hz = theta
    h = torch.stack([hx, hy, hz])
    S0 = torch.as_tensor(s0, dtype=torch.float64).reshape(nf, N, N, 3)

    def rhs(S):
        nn = (torch.roll(S, -1, 1) + torch.roll(S, 1, 1) + torch.roll(S, 1, 2) +
              torch.roll(S, -1, 2))
        nnn = (torch.roll(S, (-1, -1), (1, 2)) + torch.roll(S, (-1, 1), (1, 2)) +
               torch.roll(S, (1, -1), (1, 2)) + torch.roll(S, (1, 1), (1, 2)))
        H = J1 * nn + J2 * nnn + h
        tau = torch.cross(H, S, dim=-1)
        g = 1.0 / (1.0 + al * al)
        return g * (tau + al * torch.cross(S, tau, dim=-1))

    M = N * N
    q = 2.0 * math.pi * vx / N
    idx = torch.arange(M, dtype=torch.float64)
    th = q * torch.div(idx, N, rounding_mode="floor") + q * (idx % N)
    u = torch.exp(-1j * th)

    def fsum(Y, ph):  # sum_i ph_i Y[f, i, c] -> [f, c]
        return torch.einsum("i,fic->fc", ph, Y.reshape(nf, M, 3).to(torch.complex128))

    G = fsum(S0, torch.conj(u))
    Z = G.mean(dim=0)
    y = S0
    loss = torch.zeros((), dtype=torch.float64)
    E = nsteps // stride
    for n in range(1, nsteps + 1):
        k1 = dt * rhs(y)
        k2 = dt * rhs(y + k1 / 2)
        k3 = dt * rhs(y + k2 / 2)
        k4 = dt * rhs(y + k3)
        v = y + k1 / 6 + k2 / 3 + k3 / 3 + k4 / 6
        y = spin_len * v / torch.linalg.norm(v, dim=-1, keepdim=True)
        if n % stride == 0 and n // stride <= E:
            F = fsum(y, u)
            S = (F * (G - Z)).sum() / (M * nf)
            loss = loss + torch.abs(S - complex(target[n // stride - 1])) ** 2
    return loss / E


def test_adjoint_matches_torch_fp64_reference():
    import torch

    N, nf, dt, nsteps, stride, ck = 6, 3, 0.02, 12, 3, 5
    theta0 = [0.9, -0.2, 0.1, 0.05, -0.1, 0.2]
    s0 = asd.random_spins(N, nf, seed=4)
    rng = np.random.default_rng(1)
    E = nsteps // stride
    target = rng.normal(size=E) + 1j * rng.normal(size=E)
    p = asd.Params.make(N, nf, J1=theta0[0], J2=theta0[1], alpha=theta0[2], h=theta0[3:], dt=dt,
                        vx=1, vy=1)
    with asd.Context(p, modes=["fp64"]) as ctx:
        ctx.set_spins(s0, as_origin=True)
        loss, grad, sqt = ctx.loss_grad(nsteps, stride, ck, target)
    theta = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
    ref = torch_loss(theta, s0, N, nf, dt, nsteps, stride, 1, target)
    ref.backward()
    assert abs(loss - ref.item()) < 1e-12 * max(1.0, abs(ref.item()))
    np.testing.assert_allclose(grad, theta.grad.numpy(), rtol=1e-9, atol=1e-12)


def test_checkpoint_interval_does_not_change_the_gradient():
    N, nf, nsteps, stride = 8, 4, 20, 4
    s0 = asd.random_spins(N, nf, seed=5)
    p = asd.Params.make(N, nf, J1=1.0, J2=0.1, alpha=0.2, h=(0.1, 0.0, 0.3), dt=0.02)
    target = np.linspace(0.1, 0.5, nsteps // stride) + 0.05j
    with asd.Context(p, modes=["fp64"]) as ctx:
        ctx.set_spins(s0, as_origin=True)
        ref = ctx.loss_grad(nsteps, stride, nsteps, target)
        for ck in (1, 3, 7):
            got = ctx.loss_grad(nsteps, stride, ck, target)
            assert got[0] == ref[0]
            assert np.array_equal(got[1], ref[1])


def test_llg_kernel_does_not_change_the_gradient():
    """The forward pass and the segment recomputation step with the one-launch
    kernel or the stage kernels (asd_ctx_set_llg_kernel; the default picks by
    size): the same states bit for bit, so the same loss, gradient and S(q,t)."""
    N, nf, nsteps, stride = 20, 12, 24, 4
    s0 = asd.random_spins(N, nf, seed=6)
    p = asd.Params.make(N, nf, J1=1.0, J2=-0.2, alpha=0.1, h=(0.0, 0.1, 0.2), dt=0.02)
    target = np.linspace(0.2, 0.6, nsteps // stride) - 0.1j
    with asd.Context(p, modes=["fp64"]) as ctx:
        ctx.set_spins(s0, as_origin=True)
        got = {}
        for kern in ("fused", "stages", "auto"):
            ctx.set_llg_kernel(kern)
            got[kern] = ctx.loss_grad(nsteps, stride, 5, target)
        for kern in ("stages", "auto"):
            assert got[kern][0] == got["fused"][0]
            assert np.array_equal(got[kern][1], got["fused"][1])
            assert np.array_equal(got[kern][2], got["fused"][2])


def test_differentiation_configuration_finite_differences():
    N, nf, nsteps, stride, ck, dt = 64, 100, 1000, 10, 50, 0.01
    s0 = asd.random_spins(N, nf, seed=0)
    base = asd.Params.make(N, nf, J1=1.0, alpha=0.1, h=(0.0, 0.0, 0.2), dt=dt)
    with asd.Context(base, modes=["fp64"]) as ctx:
        ctx.set_spins(s0, as_origin=True)
        _, _, target = ctx.loss_grad(nsteps, stride, ck, None)
        theta0 = np.array([0.8, 0.0, 0.15, 0.0, 0.0, 0.0])

        def at(th):
            return asd.Params.make(N, nf, J1=th[0], J2=th[1], alpha=th[2], h=th[3:], dt=dt)

        ctx.set_params(at(theta0))
        loss, grad, _ = ctx.loss_grad(nsteps, stride, ck, target)
        assert loss > 0
        fd = np.zeros(6)
        for q in range(6):
            eps = 1e-5
            tp, tm = theta0.copy(), theta0.copy()
            tp[q] += eps
            tm[q] -= eps
            ctx.set_params(at(tp))
            lp = ctx.loss_grad(nsteps, stride, ck, target)[0]
            ctx.set_params(at(tm))
            lm = ctx.loss_grad(nsteps, stride, ck, target)[0]
            fd[q] = (lp - lm) / (2 * eps)
    scale = np.abs(fd).max()
    for q in range(6):
        assert abs(grad[q] - fd[q]) <= 1e-4 * max(abs(fd[q]), 1e-3 * scale), (q, grad[q], fd[q])


def test_autograd_wrapper_and_descent():
    import torch

    from asd_b200.autograd import sqt_loss

    N, nf, nsteps, stride, ck = 16, 8, 60, 6, 20
    s0 = asd.random_spins(N, nf, seed=2)
    truth = asd.Params.make(N, nf, J1=1.0, alpha=0.1, h=(0.0, 0.0, 0.2), dt=0.01)
    with asd.Context(truth, modes=["fp64"]) as ctx:
        ctx.set_spins(s0, as_origin=True)
        _, _, target = ctx.loss_grad(nsteps, stride, ck, None)
        theta = torch.tensor([0.8, 0.0, 0.15, 0.0, 0.0, 0.0], dtype=torch.float64,
                             requires_grad=True)
        loss = sqt_loss(theta, ctx, nsteps, stride, ck, target)
        loss.backward()
        direct = ctx.loss_grad(nsteps, stride, ck, target)[1]
        np.testing.assert_allclose(theta.grad.numpy(), direct, rtol=0, atol=0)
        losses = [loss.item()]
        opt = torch.optim.Adam([theta], lr=0.02)
        for _ in range(5):
            opt.zero_grad()
            l = sqt_loss(theta, ctx, nsteps, stride, ck, target)
            l.backward()
            opt.step()
            losses.append(l.item())
        assert losses[-1] < losses[0]


def test_forward_pays_no_adjoint_and_backward_matches():
    """asd_ctx_loss_forward runs the forward pass only (its launch count is
    that of the steps and the S(q,t) evaluations); asd_ctx_loss_backward from
    its tape gives asd_ctx_loss_grad's gradient bit for bit and
    dL/dtarget = -2 (S - target) / E; a parameter change invalidates the tape."""
    N, nf, nsteps, stride, ck = 16, 8, 60, 6, 20
    s0 = asd.random_spins(N, nf, seed=4)
    p = asd.Params.make(N, nf, J1=1.0, alpha=0.1, h=(0.0, 0.0, 0.2), dt=0.01)
    with asd.Context(p, modes=["fp64"]) as ctx:
        ctx.set_spins(s0, as_origin=True)
        _, _, target = ctx.loss_grad(nsteps, stride, ck, None)
        target = target * (1.0 + 0.01j)
        loss_ref, grad_ref, S_ref = ctx.loss_grad(nsteps, stride, ck, target)
        loss, S = ctx.loss_forward(nsteps, stride, ck, target)
        fwd_launches = ctx.last_launches()
        assert loss == loss_ref
        assert np.array_equal(S, S_ref)
        E = nsteps // stride
        # one launch per step (the one-launch RK4 step or 4 stage kernels) and
        # two per S(q,t) evaluation, plus the origin's sums: no adjoint
        assert fwd_launches <= 4 * nsteps + 2 * E + 2
        grad, dtarget = ctx.loss_backward(target)
        # the adjoint's launches come here: per step at least the segment's
        # recomputed forward step (4 stage kernels) and 5 adjoint launches
        assert ctx.last_launches() >= 9 * nsteps
        np.testing.assert_array_equal(grad, grad_ref)
        np.testing.assert_allclose(dtarget, -2.0 * (S - target) / E, rtol=1e-15, atol=0)
        grad2, _ = ctx.loss_backward(target)  # the tape stays until the next forward pass
        np.testing.assert_array_equal(grad2, grad_ref)
        ctx.set_params(asd.Params.make(N, nf, J1=1.1, alpha=0.1, h=(0.0, 0.0, 0.2), dt=0.01))
        with pytest.raises(asd.AsdError) as e:
            ctx.loss_backward(target)
        assert e.value.code == asd.ASD_ERR_STATE


def test_autograd_target_gradient():
    """With a target tensor that requires grad, backward gives dL/dtarget too."""
    import torch

    from asd_b200.autograd import sqt_loss

    N, nf, nsteps, stride, ck = 12, 6, 40, 5, 20
    s0 = asd.random_spins(N, nf, seed=5)
    p = asd.Params.make(N, nf, J1=1.0, alpha=0.1, dt=0.01)
    with asd.Context(p, modes=["fp64"]) as ctx:
        ctx.set_spins(s0, as_origin=True)
        _, _, tgt = ctx.loss_grad(nsteps, stride, ck, None)
        target = torch.tensor(tgt * 0.9, dtype=torch.complex128, requires_grad=True)
        theta = torch.tensor([1.0, 0.0, 0.1, 0.0, 0.0, 0.0], dtype=torch.float64,
                             requires_grad=True)
        loss = sqt_loss(theta, ctx, nsteps, stride, ck, target)
        loss.backward()
        S = torch.tensor(tgt, dtype=torch.complex128)
        want = -2.0 * (S - target.detach()) / (nsteps // stride)
        torch.testing.assert_close(target.grad, want, rtol=1e-14, atol=1e-16)
        # torch's own autograd of the same loss on the same S gives the same
        t2 = target.detach().clone().requires_grad_(True)
        ((S - t2).abs() ** 2).mean().backward()
        torch.testing.assert_close(target.grad, t2.grad, rtol=1e-14, atol=1e-16)
