"""getrates as a differentiable torch operation.

Forward: the CUDA getrates kernel (FP64 or mixed) through the C ABI.
Backward: the analytic adjoint kernel (chemgen_getrates_vjp), which returns
dL/dP, dL/dT and dL/dY from dL/dwdot without forming the Jacobian.
"""
from __future__ import annotations

import torch

from .runtime import GpuMechanism


class Getrates(torch.autograd.Function):
    """wdot = getrates(P, T, Y) with an analytic backward."""

    @staticmethod
    def forward(ctx, gm: GpuMechanism, P, T, Y, mode: str = "fp64"):
        P, T, Y = P.contiguous(), T.contiguous(), Y.contiguous()
        ctx.gm = gm
        ctx.save_for_backward(P, T, Y)
        return gm.getrates(P, T, Y, mode=mode)

    @staticmethod
    def backward(ctx, g):
        P, T, Y = ctx.saved_tensors
        gT, gY, gP = ctx.gm.vjp(P, T, Y, g.contiguous())
        return None, gP, gT, gY, None


def getrates(gm: GpuMechanism, P, T, Y, mode: str = "fp64"):
    """Differentiable getrates on CUDA float64 tensors (Y is [ns, ng])."""
    return Getrates.apply(gm, P, T, Y, mode)
