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
    def forward(ctx, gm: GpuMechanism, P, T, Y, mode: str = "fp64", layout: str = "species_major"):
        if layout not in ("species_major", "point_major"):
            raise ValueError("layout must be 'species_major' or 'point_major'")
        P, T = P.contiguous(), T.contiguous()
        Ys = Y.t().contiguous() if layout == "point_major" else Y.contiguous()
        ctx.gm = gm
        ctx.layout = layout
        ctx.save_for_backward(P, T, Ys)
        w = gm.getrates(P, T, Ys, mode=mode)
        return w.t().contiguous() if layout == "point_major" else w

    @staticmethod
    def backward(ctx, g):
        P, T, Ys = ctx.saved_tensors
        gs = g.t().contiguous() if ctx.layout == "point_major" else g.contiguous()
        gT, gY, gP = ctx.gm.vjp(P, T, Ys, gs)
        if ctx.layout == "point_major":
            gY = gY.t().contiguous()
        return None, gP, gT, gY, None, None


GetratesFn = Getrates


def getrates(gm: GpuMechanism, P, T, Y, mode: str = "fp64", layout: str = "species_major"):
    """Differentiable getrates on CUDA float64 tensors: Y [ns, ng] (or
    [ng, ns] with layout="point_major"), wdot in the same layout."""
    return Getrates.apply(gm, P, T, Y, mode, layout)
