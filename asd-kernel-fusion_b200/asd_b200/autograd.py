"""torch.autograd.Function over the library's adjoint (asd_ctx_loss_grad).

    theta = torch.tensor([J1, J2, alpha, hx, hy, hz], dtype=torch.float64, requires_grad=True)
    loss = sqt_loss(theta, ctx, nsteps=1000, stride=10, checkpoint=50, target=target)
    loss.backward()            # theta.grad = dL/dtheta from the adjoint RK4

The forward runs the RK4 steps and S(q,t) on the GPU and the adjoint right
away (with checkpoints every `checkpoint` steps); backward only scales the
stored gradient.  PyTorch is used for nothing else.
"""
from __future__ import annotations

import torch

from . import Context, Params

PARAM_NAMES = ("J1", "J2", "alpha", "hx", "hy", "hz")


def params_with(base: Params, theta) -> Params:
    v = [float(x) for x in theta]
    return Params(base.N, base.nfile, v[0], v[1], v[2], v[3], v[4], v[5], base.dt,
                  base.spin_len, base.vx, base.vy)


class SqtLoss(torch.autograd.Function):
    @staticmethod
    def forward(fctx, theta, context: Context, nsteps: int, stride: int, checkpoint: int, target):
        context.set_params(params_with(context.params, theta.detach().cpu().tolist()))
        loss, grad, _ = context.loss_grad(nsteps, stride, checkpoint, target)
        fctx.save_for_backward(torch.as_tensor(grad, dtype=theta.dtype, device=theta.device))
        return torch.as_tensor(loss, dtype=theta.dtype, device=theta.device)

    @staticmethod
    def backward(fctx, g):
        (grad,) = fctx.saved_tensors
        return g * grad, None, None, None, None, None


def sqt_loss(theta, context: Context, nsteps: int, stride: int, checkpoint: int, target):
    """L(theta) = mean_e |S(q, t_e; theta) - target_e|^2, differentiable in theta."""
    return SqtLoss.apply(theta, context, int(nsteps), int(stride), int(checkpoint), target)
