"""torch.autograd.Function around the adjoint of the summed keypoint maps.

For checking the hand-written adjoint (bimp_adjoint_*, include/bimp_b200_adjoint.h)
against finite differences and the FP64 CPU reference gradient with torch's
own machinery.  The loss is

    L = sum_i sum_s sum_{y,x} M_is[y,x] * D_is[y,x]

for float images X (n, H, W) and parameters theta = (alpha, rho, w_tan, w_rad):
the wavelength scale factor, the sigma ratio and the two inhibition weights.
The library evaluates the forward at the bank's parameters only (the filter
bank is built for them), so theta must equal the Adjoint's nominal values;
its gradient is the derivative there.

    adj = api.Adjoint(W, H, n, lambdas)
    theta = summed_map_theta(adj, requires_grad=True)
    loss = summed_map_loss(images, theta, masks, adj)
    loss.backward()            # images.grad, theta.grad
"""
from __future__ import annotations

import torch

from . import api


def summed_map_theta(adj: "api.Adjoint", requires_grad: bool = True) -> torch.Tensor:
    """The nominal (alpha, rho, w_tan, w_rad) of an Adjoint, float64 on its device."""
    p = adj.params
    return torch.tensor([1.0, p.sigma_ratio, p.w_tan, p.w_rad], dtype=torch.float64, device="cuda",
                        requires_grad=requires_grad)


class SummedKeypointMapLoss(torch.autograd.Function):
    """forward(images, theta, masks, adj) -> L (float64 scalar on the device);
    backward -> (dL/dimages, dL/dtheta)."""

    @staticmethod
    def forward(ctx, images, theta, masks, adj):
        nominal = summed_map_theta(adj, requires_grad=False)
        if not torch.equal(theta.detach().to(nominal), nominal):
            raise ValueError("theta must equal the Adjoint's nominal (alpha, rho, w_tan, w_rad)")
        loss = adj.forward(images.detach().contiguous(), masks.detach().contiguous())
        ctx.adj = adj
        ctx.theta_dtype = theta.dtype
        return loss.reshape(()).clone()

    @staticmethod
    def backward(ctx, grad_out):
        g, gp = ctx.adj.backward()
        go = grad_out.to(torch.float64)
        return (g * go.to(g.dtype)).clone(), (gp * go).to(ctx.theta_dtype), None, None


def summed_map_loss(images: torch.Tensor, theta: torch.Tensor, masks: torch.Tensor, adj: "api.Adjoint"):
    return SummedKeypointMapLoss.apply(images, theta, masks, adj)
