"""The GP loss as a differentiable torch function of the hyper-parameters.

``nlml(gp, hyper)`` returns the negative log marginal likelihood per point
that the reference's ``calculate_loss`` returns (core/src/cpu/gp_functions.cpp:
730-781, 0.5*(y^T alpha + log det K + n log 2 pi)/n), as a torch scalar whose
backward pass is the adjoint gradient computed on the GPU in the same
factorisation (no extra pass, no finite differences):

    dL/dtheta_p = 0.5/n * (tr(K^-1 dK/dtheta_p) - alpha^T dK/dtheta_p alpha)

with theta = (lengthscale, vertical_lengthscale, noise_variance) in the
constrained (positive) parameterisation the reference's GP API takes.  The
library's kernel returns the gradient the reference's optimiser uses, with
respect to the unconstrained parameters u (theta = softplus(u), +1e-6 for the
noise; core/src/cpu/gp_optimizer.cpp:12-36, tiled_algorithms.cpp:296-426),
i.e. scaled by dtheta/du = sigmoid(u) = 1 - exp(-theta); this module divides
that factor out.
"""
from __future__ import annotations

import math

import torch

from . import capi

_NOISE_JITTER = 1e-6  # to_constrained adds it to the noise (gp_optimizer.cpp:12-22)


def _dtheta_du(theta: float, noise: bool) -> float:
    """sigmoid(softplus^-1(theta)) = 1 - exp(-theta) (theta - 1e-6 for the noise)."""
    t = theta - _NOISE_JITTER if noise else theta
    return -math.expm1(-t)


class GPLoss(torch.autograd.Function):
    """loss = nlml(theta) for one device-resident GP (a ``capi.CudaGP``)."""

    @staticmethod
    def forward(ctx, hyper: torch.Tensor, gp: "capi.CudaGP") -> torch.Tensor:
        h = [float(v) for v in hyper.detach().to("cpu", torch.float64).reshape(3)]
        ctx.in_dtype, ctx.in_shape = hyper.dtype, hyper.shape
        if ctx.needs_input_grad[0]:
            loss, g_u = gp.loss_grad(h)
            g = [g_u[p] / _dtheta_du(h[p], p == 2) for p in range(3)]
            ctx.save_for_backward(torch.tensor(g, dtype=torch.float64, device=hyper.device))
        else:
            loss = gp.compute_loss(h)
        return torch.tensor(loss, dtype=torch.float64, device=hyper.device)

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        (g,) = ctx.saved_tensors
        return (grad_out * g).to(ctx.in_dtype).reshape(ctx.in_shape), None


def nlml(gp: "capi.CudaGP", hyper: torch.Tensor) -> torch.Tensor:
    """Differentiable loss of ``gp`` at ``hyper`` = (lengthscale, vertical_lengthscale, noise_variance)."""
    if hyper.numel() != 3:
        raise ValueError("hyper must hold (lengthscale, vertical_lengthscale, noise_variance)")
    return GPLoss.apply(hyper, gp)
