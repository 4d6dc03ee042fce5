"""torch.autograd wrapper: B = biot_savart(xyz, w, J, targets) with gradients for the source
positions and the current densities from the hand-written adjoint FMM (fmm_adjoint).

Used for gradient checks against central differences and the FP64 direct-sum adjoint; the
weights and the target positions are treated as constants. J = None selects the reference's
azimuthal current direction perp(q)/|perp(q)| (FMM/FMMGPU/integration.cpp:155); its dependence on
the source positions is then part of the position gradient, and J has no gradient."""
from __future__ import annotations

import torch

from .solver import Plan


class _BiotSavartFMM(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xyz, w, J, targets, current, plan):
        plan.set_sources(xyz, w, J)
        plan.set_targets(targets)
        B, _ = plan.solve(current, 1)
        ctx.plan = plan
        ctx.current = current
        ctx.has_J = J is not None
        # the plan may be reused for another forward before this backward runs: keep this call's
        # inputs and the plan's input generation, and restore them in backward if they changed
        ctx.generation = plan.generation
        ctx.save_for_backward(xyz, w, J if J is not None else xyz.new_empty(0), targets)
        return B

    @staticmethod
    def backward(ctx, gB):
        plan = ctx.plan
        xyz, w, J, targets = ctx.saved_tensors
        if plan.generation != ctx.generation:
            plan.set_sources(xyz, w, J if ctx.has_J else None)
            plan.set_targets(targets)
            ctx.generation = plan.generation
        dJ, dx = plan.adjoint(gB.contiguous(), ctx.current, want_dJ=ctx.has_J)
        return dx, None, dJ if ctx.has_J else None, None, None, None


def biot_savart(xyz, w, J, targets, current=1.0, order=12, leaf_capacity=64, m2l="simt", plan=None):
    """B at `targets` from sources (xyz, w, J), all CUDA tensors of one floating type (float32 or
    float64). Differentiable in xyz and J (J = None: the azimuthal direction, differentiable in xyz)."""
    if plan is None:
        precision = "fp64" if xyz.dtype == torch.float64 else "fp32"
        plan = Plan(order=order, leaf_capacity=leaf_capacity, precision=precision,
                    m2l=m2l if precision == "fp32" else "simt", device=xyz.device.index or 0)
    return _BiotSavartFMM.apply(xyz, w, J, targets, float(current), plan)
