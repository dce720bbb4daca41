"""Differentiable tumour-growth loss for PyTorch over the C ABI.

``TumorLoss`` runs the forward solve and the hand-written discrete adjoint
(gbfk_forward_adjoint: binomial checkpointing, FP64 loss and gradient sums)
in one call and hands the gradients to autograd.  Inputs are the physical
parameters: Dw in cm^2/day (rescaled by 1/L^2 and Dg = Dw/10 as in
Glioma_ReactionDiffusion.cpp:302-303), rho in 1/day, and the initial field:
either the Gaussian of width sigma around the tumour origin x0 (unit cube) or
an explicit field c0 (a dense n^3 tensor, x fastest, like the pool's own
dense volumes).  dt and the step count are held fixed (chosen from a nominal
Dw), so the loss is a smooth function of the parameters between switches.
"""
from __future__ import annotations

import numpy as np
import torch

from .solver import BlockPool


class TumorLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, Dw, rho, x0, c0, pool: BlockPool, L_cm: float, dt: float, nsteps: int, sigma: float,
                nsnapshots: int = 64):
        R = np.float64 if pool.precision == "f64" else np.float32
        L = R(L_cm)
        Dw_r = R(R(float(Dw)) / (L * L))
        Dg_r = R(0.1 * np.float64(Dw_r))
        if c0 is not None:
            # the initial field as given: d loss / d c0 is the adjoint state at t = 0
            pool.upload_dense("phi", np.ascontiguousarray(c0.detach().cpu().numpy(), dtype=R))
            res = pool.forward_adjoint(float(Dw_r), float(Dg_r), float(R(float(rho))), dt, nsteps, sigma=0.0,
                                       nsnapshots=nsnapshots, grad_c0=True)
            g_c0 = torch.from_numpy(res["grad_c0"].astype(np.float64)).to(dtype=c0.dtype, device=c0.device)
            g_x0 = None
        else:
            res = pool.forward_adjoint(float(Dw_r), float(Dg_r), float(R(float(rho))), dt, nsteps,
                                       x0=[float(v) for v in x0.detach().cpu()], sigma=sigma,
                                       nsnapshots=nsnapshots)
            g_c0 = None
            g_x0 = torch.tensor(res["dx0"], dtype=torch.float64)
        # d/dDw_phys = d/dDw_rescaled / L^2 (Dg follows Dw)
        ctx.g_dw = torch.tensor(res["dDw"] / float(L * L), dtype=torch.float64)
        ctx.g_rho = torch.tensor(res["drho"], dtype=torch.float64)
        ctx.g_x0, ctx.g_c0 = g_x0, g_c0
        return torch.tensor(res["loss"], dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad):
        g_x0 = None if ctx.g_x0 is None else grad * ctx.g_x0
        g_c0 = None if ctx.g_c0 is None else grad.to(ctx.g_c0.dtype) * ctx.g_c0
        return grad * ctx.g_dw, grad * ctx.g_rho, g_x0, g_c0, None, None, None, None, None, None


def tumor_loss(pool: BlockPool, Dw, rho, x0, L_cm: float, dt: float, nsteps: int, sigma: float,
               nsnapshots: int = 64, c0=None):
    """Scalar loss tensor differentiable w.r.t. Dw, rho and the initial field.

    With ``c0`` None the initial field is the Gaussian of width ``sigma``
    around ``x0`` and the gradient reaches ``x0``; with ``c0`` (n^3 tensor)
    the initial field is ``c0`` itself, ``x0`` is unused and ``c0.grad`` is
    d loss / d c0."""
    return TumorLoss.apply(Dw, rho, x0, c0, pool, L_cm, dt, nsteps, sigma, nsnapshots)
