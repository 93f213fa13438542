"""2-D parallel-beam projector: drop-in for Projector2DParallelPython.

The reference's 2-D class (vamtoolbox/projector/Projector2DParallel.py:47-285)
is reached only after ``TargetGeometry.segmentZ(int)`` makes the target 2-D.
It uses the same rotate-and-sum / np.interp discretisation as the 3-D class
with one slice, plus three behaviours kept here:
  * ``forward`` clips its input to the inscribed circle in place (:161);
  * ``backward`` zeroes ``b[zero_dose_sino]`` in place before projecting (:206-207);
  * ``backward(b, clipping=False)`` skips the circle clip (:188, 230-231).
Its digitised occlusion model (:70-143, 235-247) is not provided: a 2-D
target with an attenuation field raises NotImplementedError.
(Its backward also reads ``target_geo.target``, an attribute the reference's
TargetGeometry never sets, :205; this class uses the array's shape.)
"""
from __future__ import annotations

import numpy as np
import torch

from ..util.data import clipToCircle
from .Projector3DParallel import ParallelPlan


class Projector2DParallel:
    def __init__(self, target_geo, proj_geo, device=None):
        self.target_geo = target_geo
        self.proj_geo = proj_geo
        if getattr(proj_geo, "occlusion", None) is not None or getattr(proj_geo, "attenuation_field", None) is not None:
            raise NotImplementedError("2-D occlusion (Projector2DParallel.py:70-143) is not provided; use a 3-D target")
        arr = np.asarray(target_geo.array)
        self.nY, self.nX = arr.shape[:2]
        self.angles = np.asarray(proj_geo.angles, dtype=np.float64)
        self.plan = ParallelPlan(self.nY, self.nX, 1, self.angles, device)
        self.plan_noclip = None
        self.device = self.plan.device

    def forward(self, target):
        if isinstance(target, torch.Tensor):
            x = target.reshape(self.nY, self.nX)
            outside = torch.as_tensor(~_inside(self.nY, self.nX), device=x.device)
            x[outside] = 0
            return self.plan.forward(x.to(self.device, torch.float32).reshape(self.nY, self.nX, 1).contiguous())[:, :, 0]
        x = clipToCircle(target)
        t = torch.as_tensor(np.ascontiguousarray(x, dtype=np.float32), device=self.device).reshape(self.nY, self.nX, 1)
        return self.plan.forward(t)[:, :, 0].double().cpu().numpy()

    def backward(self, b, clipping=True):
        if self.proj_geo.zero_dose_sino is not None:
            b[self.proj_geo.zero_dose_sino] = 0.0
        is_t = isinstance(b, torch.Tensor)
        t = (b if is_t else torch.as_tensor(np.ascontiguousarray(b, dtype=np.float32)))
        t = t.to(self.device, torch.float32).reshape(self.nY, self.angles.size, 1).contiguous()
        x = self.plan.backward_ref(t)[:, :, 0]
        if not clipping:
            raise NotImplementedError("backward(clipping=False) is not provided")
        return x if is_t else x.double().cpu().numpy()


def _inside(ny, nx):
    cy, cx = np.meshgrid(np.linspace(-1, 1, ny), np.linspace(-1, 1, nx))
    return ~(cx ** 2 + cy ** 2 > 1)
