"""torch.autograd.Function over the library's adjoint (asd_ctx_loss_forward /
asd_ctx_loss_backward).

    theta = torch.tensor([J1, J2, alpha, hx, hy, hz], dtype=torch.float64, requires_grad=True)
    loss = sqt_loss(theta, ctx, nsteps=1000, stride=10, checkpoint=50, target=target)
    loss.backward()            # theta.grad = dL/dtheta from the adjoint RK4

forward runs the RK4 steps and S(q,t) on the GPU and keeps the checkpoints;
backward runs the adjoint from them, so an evaluation that is never
differentiated costs the forward pass only.  The target may be a complex
tensor (or 2E real values, re/im interleaved); if it requires grad, it
receives dL/dtarget.  PyTorch is used for nothing else.
"""
from __future__ import annotations

import numpy as np
import torch

from . import Context, Params

PARAM_NAMES = ("J1", "J2", "alpha", "hx", "hy", "hz")


def params_with(base: Params, theta) -> Params:
    v = [float(x) for x in theta]
    return Params(base.N, base.nfile, v[0], v[1], v[2], v[3], v[4], v[5], base.dt,
                  base.spin_len, base.vx, base.vy)


def _target_np(target):
    if isinstance(target, torch.Tensor):
        return target.detach().cpu().numpy()
    return np.asarray(target)


class SqtLoss(torch.autograd.Function):
    @staticmethod
    def forward(fctx, theta, target, context: Context, nsteps: int, stride: int, checkpoint: int):
        context.set_params(params_with(context.params, theta.detach().cpu().tolist()))
        tnp = _target_np(target)
        loss, _ = context.loss_forward(nsteps, stride, checkpoint, tnp)
        fctx.context = context
        fctx.target = tnp
        fctx.target_meta = (target.dtype, target.device, target.shape) \
            if isinstance(target, torch.Tensor) else None
        return torch.as_tensor(loss, dtype=theta.dtype, device=theta.device)

    @staticmethod
    def backward(fctx, g):
        grad, dtarget = fctx.context.loss_backward(fctx.target)
        g_theta = g * torch.as_tensor(grad, dtype=g.dtype, device=g.device)
        g_target = None
        if fctx.target_meta is not None and fctx.needs_input_grad[1]:
            dtype, device, shape = fctx.target_meta
            if dtype.is_complex:
                d = torch.as_tensor(dtarget, device=device).to(dtype)
            else:
                d = torch.as_tensor(np.stack([dtarget.real, dtarget.imag], axis=-1).reshape(-1),
                                    dtype=dtype, device=device)
            g_target = (g * d).reshape(shape)
        return g_theta, g_target, None, None, None, None


def sqt_loss(theta, context: Context, nsteps: int, stride: int, checkpoint: int, target):
    """L(theta) = mean_e |S(q, t_e; theta) - target_e|^2, differentiable in theta
    (and in target when it is a tensor that requires grad)."""
    return SqtLoss.apply(theta, target, context, int(nsteps), int(stride), int(checkpoint))
