"""Differentiable projectors: torch.autograd.Function wrappers over the C ABI.

* :func:`parallel_forward` -- R1 forward; backward is the matched transpose
  kernel (vam_parallel_adjoint), so gradients are exact for the discretised
  operator (the reference's own backward, R2, is not its transpose).
* :func:`parallel_adjoint` -- the matched transpose; backward is R1.
* :func:`ray_integrate` -- curved-ray forward (R6) as a function of the field f
  and, optionally, of the attenuation grid alpha: d/df is the deposit kernel
  (R5, its exact transpose), d/dalpha recomputes every ray's path
  (vam_ray_grad_alpha) instead of storing it.
* :func:`ray_deposit` -- R5; backward is R6.
* :func:`vec_forward` -- the vector-geometry (ASTRA-model) forward; backward is
  its exact transpose (vam_vec_adjoint), not ASTRA's voxel-driven backprojection.
* :func:`line2d_forward` / :func:`line2d_backward` -- the 2-D line model and
  its exact transpose, each the other's gradient.

Plans are the objects of :mod:`vamtoolbox_b200.projector` (``ParallelPlan``,
``RayPlan``, ``VecPlan``, ``Line2DPlan``); inputs are float32 CUDA tensors of the plan's shapes.
"""
from __future__ import annotations

import torch


class _ParallelForward(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, plan):
        ctx.plan = plan
        return plan.forward(x.contiguous())

    @staticmethod
    def backward(ctx, gb):
        return ctx.plan.adjoint(gb.contiguous()), None


class _ParallelAdjoint(torch.autograd.Function):
    @staticmethod
    def forward(ctx, b, plan):
        ctx.plan = plan
        return plan.adjoint(b.contiguous())

    @staticmethod
    def backward(ctx, gx):
        return ctx.plan.forward(gx.contiguous()), None


def parallel_forward(x, plan):
    """Sinogram of x (differentiable)."""
    return _ParallelForward.apply(x, plan)


def parallel_adjoint(b, plan):
    """Exact transpose of parallel_forward applied to b (differentiable)."""
    return _ParallelAdjoint.apply(b, plan)


class _RayIntegrate(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f, alpha, plan, index_model, attenuation_model, absorption_model):
        if alpha is not None:
            from .medium import AttenuationModel

            am = AttenuationModel(attenuation_model.coord_vec, type="interpolation", form="freeform",
                                  alpha_x=alpha.detach(), device=alpha.device)
            plan.bind_medium(index_model, am, absorption_model)
        ctx.plan = plan
        ctx.has_alpha = alpha is not None
        ctx.save_for_backward(f)
        return plan.integrate(f)

    @staticmethod
    def backward(ctx, gg):
        (f,) = ctx.saved_tensors
        plan = ctx.plan
        gf = plan.deposit(gg.contiguous()) if ctx.needs_input_grad[0] else None
        galpha = None
        if ctx.has_alpha and ctx.needs_input_grad[1]:
            galpha = torch.zeros(plan.grid_shape, dtype=torch.float32, device=gg.device)
            plan.grad_alpha(f, gg.contiguous(), grad_att=galpha)
        return gf, galpha, None, None, None, None


def ray_integrate(f, plan, alpha=None, index_model=None, attenuation_model=None, absorption_model=None):
    """Ray integrals of f (differentiable in f and, if given, in the attenuation grid alpha).

    With alpha, the plan is re-bound to an attenuation model built from alpha
    (same grid as attenuation_model); index_model and absorption_model must be
    the models the plan was built with.
    """
    return _RayIntegrate.apply(f, alpha, plan, index_model, attenuation_model, absorption_model)


class _RayDeposit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, g, plan):
        ctx.plan = plan
        return plan.deposit(g.contiguous())

    @staticmethod
    def backward(ctx, gd):
        return ctx.plan.integrate(gd.contiguous()), None


def ray_deposit(g, plan):
    """Dose deposited by ray energies g (differentiable)."""
    return _RayDeposit.apply(g, plan)


class _VecForward(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, plan):
        ctx.plan = plan
        return plan.forward(x.contiguous())

    @staticmethod
    def backward(ctx, gb):
        return ctx.plan.adjoint(gb.contiguous()), None


def vec_forward(x, plan):
    """Vector-geometry sinogram of x (differentiable; gradient by the exact transpose)."""
    return _VecForward.apply(x, plan)


class _Line2DForward(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, plan):
        ctx.plan = plan
        return plan.forward(x)

    @staticmethod
    def backward(ctx, gb):
        return ctx.plan.backward(gb.contiguous()), None


class _Line2DBackward(torch.autograd.Function):
    @staticmethod
    def forward(ctx, b, plan):
        ctx.plan = plan
        return plan.backward(b)

    @staticmethod
    def backward(ctx, gx):
        return ctx.plan.forward(gx.contiguous()), None


def line2d_forward(x, plan):
    """2-D line-model sinogram of x (differentiable)."""
    return _Line2DForward.apply(x, plan)


def line2d_backward(b, plan):
    """Exact transpose of line2d_forward applied to b (differentiable)."""
    return _Line2DBackward.apply(b, plan)
