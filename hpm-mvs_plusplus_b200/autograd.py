"""torch.autograd binding of the differentiable bilateral NCC (hpm_eval_cost_grad).

    cost = NCCCost.apply(theta, ctx, ref, srcs, params, px)

theta is an (n, 3) float tensor of (depth, nx, ny) per pixel in the reference
camera frame (nz = -sqrt(1 - nx^2 - ny^2)); the result is the (n, S) tensor of
per-view costs.  The forward pass asks the library for the costs and their
gradients in one call (the adjoint kernel recomputes the warped samples); the
backward pass contracts the stored (n, S, 3) Jacobian with the incoming
gradient.  CUDA tensors stay on the device (hpm_eval_cost_grad_device); host
tensors go through hpm_eval_cost_grad.
"""
from __future__ import annotations

import numpy as np
import torch


class NCCCost(torch.autograd.Function):
    @staticmethod
    def forward(fctx, theta: torch.Tensor, hctx, ref: int, srcs, params, px):
        if theta.is_cuda:
            p = px if torch.is_tensor(px) else torch.as_tensor(np.asarray(px), device=theta.device)
            cost, grad = hctx.eval_cost_grad_tensors(ref, srcs, params, p.to(theta.device), theta.detach())
            fctx.save_for_backward(grad)
            return cost.to(theta.dtype)
        th = theta.detach().to("cpu", torch.float32).numpy()
        p = px.cpu().numpy() if torch.is_tensor(px) else np.asarray(px)
        cost, grad = hctx.eval_cost_grad(ref, srcs, params, p, th, with_grad=True)
        fctx.save_for_backward(torch.from_numpy(grad))
        return torch.from_numpy(cost).to(dtype=theta.dtype)

    @staticmethod
    def backward(fctx, grad_out: torch.Tensor):
        (jac,) = fctx.saved_tensors
        g = (grad_out.to(jac.dtype).unsqueeze(-1) * jac).sum(dim=1)
        return g.to(grad_out.dtype), None, None, None, None, None
