"""2-D parallel-beam projector: drop-in for Projector2DParallelPython.

The reference's 2-D class (vamtoolbox/projector/Projector2DParallel.py:47-285)
is reached only after ``TargetGeometry.segmentZ(int)`` makes the target 2-D.
It uses the same rotate-and-sum / np.interp discretisation as the 3-D class
with one slice, plus these behaviours, kept here:
  * ``forward`` clips its input to the inscribed circle in place (:161);
  * ``backward`` zeroes ``b[zero_dose_sino]`` in place before projecting (:206-207);
  * ``backward(b, clipping=False)`` skips the circle clip (:188, 230-231);
  * ``proj_geo.occlusion`` (a boolean [nY, nX] mask) selects the digitised
    occlusion (:70-143): per angle the least s = x sin + y cos of the
    occluded pixels in each np.digitize bin of t = x cos - y sin, built on
    the device; the forward zeroes samples past their column's minimum
    (:177-182) and the backward pixels whose s exceeds the minimum of their
    t's bin (:220-222, 235-247).  The attenuation field, like in the
    reference's 2-D class, only selects this class; it is not a shadow.
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
        arr = np.asarray(target_geo.array)
        self.nY, self.nX = arr.shape[:2]
        self.angles = np.asarray(proj_geo.angles, dtype=np.float64)
        self.plan = ParallelPlan(self.nY, self.nX, 1, self.angles, device)
        self.occlusion = getattr(proj_geo, "occlusion", None)
        if self.occlusion is not None:
            self.plan.set_occlusion_2d(np.asarray(self.occlusion, dtype=bool))
        self.device = self.plan.device

    @property
    def occ_sinogram(self):
        """The occlusion sinogram [nY, n_angles] (float64, NaN where a bin holds no occluded pixel), as
        the reference's ``occ_sinogram`` attribute; None without an occlusion."""
        if self.occlusion is None:
            return None
        return self.plan.occlusion_sinogram_2d().cpu().numpy()

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
        x = (self.plan.backward_ref(t) if clipping else self.plan.backward_ref_noclip(t))[:, :, 0]
        return x if is_t else x.double().cpu().numpy()


def _inside(ny, nx):
    cy, cx = np.meshgrid(np.linspace(-1, 1, ny), np.linspace(-1, 1, nx))
    return ~(cx ** 2 + cy ** 2 > 1)


# The reference's names for the same dispatch slots (projectorconstructor.py:74-160).  The
# ASTRA-model CUDA class (the 2-D line projector) is projector/Projector2DParallelCUDA.py.
Projector2DParallelPython = Projector2DParallel
Projector2DParallelAstra = Projector2DParallel
