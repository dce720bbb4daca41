"""Differentiable tumour-growth loss for PyTorch over the C ABI.

``TumorLoss`` runs the forward solve and the hand-written discrete adjoint
(gbfk_forward_adjoint: binomial checkpointing, FP64 loss and gradient sums)
in one call and hands the gradients to autograd.  Inputs are the physical
parameters: Dw in cm^2/day (rescaled by 1/L^2 and Dg = Dw/10 as in
Glioma_ReactionDiffusion.cpp:302-303), rho in 1/day and the tumour origin x0 in
the unit cube.  dt and the step count are held fixed (chosen from a nominal
Dw), so the loss is a smooth function of the parameters between switches.
"""
from __future__ import annotations

import numpy as np
import torch

from .solver import BlockPool


class TumorLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, Dw, rho, x0, pool: BlockPool, L_cm: float, dt: float, nsteps: int, sigma: float,
                nsnapshots: int = 64):
        R = np.float64 if pool.precision == "f64" else np.float32
        L = R(L_cm)
        Dw_r = R(R(float(Dw)) / (L * L))
        Dg_r = R(0.1 * np.float64(Dw_r))
        res = pool.forward_adjoint(float(Dw_r), float(Dg_r), float(R(float(rho))), dt, nsteps,
                                   x0=[float(v) for v in x0.detach().cpu()], sigma=sigma, nsnapshots=nsnapshots)
        # d/dDw_phys = d/dDw_rescaled / L^2 (Dg follows Dw)
        g_dw = torch.tensor(res["dDw"] / float(L * L), dtype=torch.float64)
        g_rho = torch.tensor(res["drho"], dtype=torch.float64)
        g_x0 = torch.tensor(res["dx0"], dtype=torch.float64)
        ctx.save_for_backward(g_dw, g_rho, g_x0)
        return torch.tensor(res["loss"], dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad):
        g_dw, g_rho, g_x0 = ctx.saved_tensors
        return grad * g_dw, grad * g_rho, grad * g_x0, None, None, None, None, None, None


def tumor_loss(pool: BlockPool, Dw, rho, x0, L_cm: float, dt: float, nsteps: int, sigma: float,
               nsnapshots: int = 64):
    """Scalar loss tensor differentiable w.r.t. Dw, rho and x0 (torch tensors)."""
    return TumorLoss.apply(Dw, rho, x0, pool, L_cm, dt, nsteps, sigma, nsnapshots)
