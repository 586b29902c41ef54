"""The torch.autograd.Function of the adjoint calibration loss.

`GPKLoss.apply(problem, eigenstrain, anisotropy, mobility)` returns the
FP64 loss of an :class:`gpk.adjoint.AdjointProblem` (interface-velocity
misfit plus elastic energy at a fixed label map) as a 0-d tensor.  Its
forward runs one forward pass of the model in libgpk_b200.so; its backward
re-runs the forward (nothing is kept between the two: the spectral buffers
are recomputed, not stored) and the hand-written discrete adjoint, and
returns the gradients for the three in-plane eigenstrain components, the
four anisotropy coefficients and the per-grain mobilities.  The reference
(albert-hzbn/GPK) has no derivative code; the gradients are checked against
FP64 central differences of the forward.
"""
from __future__ import annotations

import torch

from .adjoint import AdjointProblem


class GPKLoss(torch.autograd.Function):
    """loss = GPKLoss.apply(problem, eigenstrain (3), anisotropy (4), mobility (n_mob)), float64."""

    @staticmethod
    def forward(ctx, problem: AdjointProblem, eig, aniso, mob):
        theta = torch.cat([eig.detach(), aniso.detach(), mob.detach()]).cpu().numpy()
        ctx.problem = problem
        ctx.save_for_backward(eig, aniso, mob)
        return torch.tensor(problem.forward(theta), dtype=torch.float64, device=eig.device)

    @staticmethod
    def backward(ctx, grad_out):
        eig, aniso, mob = ctx.saved_tensors
        theta = torch.cat([eig.detach(), aniso.detach(), mob.detach()]).cpu().numpy()
        _, g = ctx.problem.gradient(theta)
        g = torch.from_numpy(g).to(device=eig.device, dtype=torch.float64) * grad_out
        return None, g[:3], g[3:7], g[7:]


def gpk_loss(problem: AdjointProblem, eig, aniso, mob):
    """Differentiable loss of `problem` at (eigenstrain, anisotropy, mobility)."""
    return GPKLoss.apply(problem, eig, aniso, mob)
