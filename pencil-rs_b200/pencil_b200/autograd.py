"""torch.autograd wrappers over the library's transforms.

Forward passes run the plan's FORWARD / INVERSE / BACKWARD kernels; backward
passes run the hand-written adjoint kernels (PB_VJP_*), so gradients never go
through a library FFT.  Complex gradients follow torch's convention
(dL/dRe + i dL/dIm), which is the adjoint under the real inner product that
the VJP kernels implement.  The transforms are linear, so nothing is saved
for backward except the plan.
"""

from __future__ import annotations

import torch

from . import _lib as L


class _PlanOp(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, plan, op, vjp_op):
        ctx.plan, ctx.vjp_op = plan, vjp_op
        fwd_like = op in (L.FORWARD, L.VJP_INVERSE, L.VJP_BACKWARD)
        out_dtype = plan.output_dtype if fwd_like else plan.input_dtype
        out_n = plan.info.output_elems if fwd_like else plan.info.input_elems
        out = torch.empty(out_n, dtype=out_dtype, device=x.device)
        plan.execute(op, x.contiguous(), out, check_spectrum=(op != L.FORWARD) and plan._reverse_checks)
        return out

    @staticmethod
    def backward(ctx, g):
        plan = ctx.plan
        vjp_fwd_like = ctx.vjp_op in (L.FORWARD, L.VJP_INVERSE, L.VJP_BACKWARD)
        n = plan.info.output_elems if vjp_fwd_like else plan.info.input_elems
        dtype = plan.output_dtype if vjp_fwd_like else plan.input_dtype
        gin = torch.empty(n, dtype=dtype, device=g.device)
        plan.execute(ctx.vjp_op, g.contiguous(), gin)
        return gin, None, None, None


def forward(plan, x):
    """plan.forward with the adjoint kernel as its backward."""
    return _PlanOp.apply(x, plan, L.FORWARD, L.VJP_FORWARD)


def inverse(plan, x):
    """plan.inverse (normalised) with the adjoint kernel as its backward."""
    return _PlanOp.apply(x, plan, L.INVERSE, L.VJP_INVERSE)


def backward(plan, x):
    """plan.backward (raw) with the adjoint kernel as its backward."""
    return _PlanOp.apply(x, plan, L.BACKWARD, L.VJP_BACKWARD)


class _Spectral(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, plan, mode, scale):
        ctx.plan, ctx.mode, ctx.scale = plan, mode, scale
        out = torch.empty_like(x)
        plan.spectral_multiply(mode, scale, x.contiguous(), out)
        return out

    @staticmethod
    def backward(ctx, g):
        # a real diagonal multiplier is its own adjoint
        out = torch.empty_like(g)
        ctx.plan.spectral_multiply(ctx.mode, ctx.scale, g.contiguous(), out)
        return out, None, None, None


def spectral_multiply(plan, x, mode="poisson", scale=1.0):
    """m(k) * x on the plan's spectral layout: "k2" (|k|^2) or "poisson" (-1/|k|^2, 0 at k=0)."""
    m = {"k2": 0, "poisson": 1}[mode]
    return _Spectral.apply(x, plan, m, float(scale))
