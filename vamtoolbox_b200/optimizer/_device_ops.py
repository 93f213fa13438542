"""The projector entry points the fused optimizer engines run on the device.

``device_ops(P, target_geo, n_iter)`` returns (back(b, out), fwd(x, out), volume shape, sinogram shape,
device) for a projector of this package -- the parallel-beam plan (with the reference's zero-dose
step before every backprojection), the ray tracer (deposit / integrate, its trajectory cache filled
once for runs of several iterations), the vector-geometry projector, the algebraic propagator -- or
None when the projector has no device entry points.  Each call writes into ``out`` on the current
stream and allocates nothing, so an engine captures its iteration as one CUDA graph.
"""
from __future__ import annotations

import numpy as np


def device_ops(P, target_geo, n_iter=1):
    plan = getattr(P, "plan", None)
    if plan is not None and hasattr(plan, "backward_ref"):
        # the zero-dose entries of b are set to 0 before every backprojection, as the reference's projector
        # does (no-op without a zero-dose region; the mask is built now, before any capture)
        zd = getattr(P, "zero_dose_", lambda t: t)
        if hasattr(P, "zero_dose_mask"):
            P.zero_dose_mask()
        return (lambda b, out: plan.backward_ref(zd(b), out), lambda x, out: plan.forward(x, out),
                plan.shape_vol, plan.shape_sino, P.device)
    if plan is not None and hasattr(plan, "deposit"):
        # the ray paths depend on the medium only: trace them once for the whole run when the cache fits
        # (half of the free device memory), before any capture
        if n_iter > 1 and not getattr(plan, "has_trajectories", True):
            plan.prepare_trajectories()
        return (lambda b, out: plan.deposit(b, out), lambda x, out: plan.integrate(x, out),
                plan.grid_shape, (plan.num_rays,), P.device)
    if plan is not None and hasattr(P, "backward_t") and hasattr(P, "forward_t"):
        # vector-geometry (ASTRA-model) projector: its wrappers carry the circle clip and mask
        return (lambda b, out: P.backward_t(b, out), lambda x, out: P.forward_t(x, out),
                plan.shape_vol, plan.shape_sino, P.device)
    from ..projector.pyTorchAlgebraicPropagation import PyTorchAlgebraicPropagator

    if isinstance(P, PyTorchAlgebraicPropagator):
        # algebraic propagator: its CSR products (z-tiled) into the iteration's buffers
        return (lambda b, out: P.backward_t(b, out), lambda x, out: P.forward_t(x, out),
                tuple(np.shape(target_geo.array)), (P.n_row_eff,), P.device)
    return None
