"""2-D parallel beam with ASTRA's "line" model: drop-in for the reference's
``Projector2DParallelCUDAAstra`` (vamtoolbox/projector/Projector2DParallelCUDA.py:7-45).

The reference builds an ASTRA ``line`` projector for a ``parallel`` geometry
(detector width nX, unit spacing) and calls ``create_sino`` /
``create_backprojection`` with it.  Here the same model runs on
libvamcore's ``vam_line2d_*`` kernels: the weight of a (ray, pixel) pair is
the length of the ray (a zero-width line) inside the unit pixel, in ASTRA's
2-D frame (row 0 on top, detector centred, rays along (sin a, -cos a)); the
backprojection is the forward's exact transpose.  ASTRA is not available to
pin against; at equal angles this model agrees with the reference-pinned
Python projector to 0.4 % (relative L2, after the two centring conventions),
which fixes its orientation.  Selected for 2-D targets with
``ProjectionGeometry(..., parallel_model="astra")``.

Image [nY][nX] -> sinogram [nT = nX][nA].  numpy in -> float64 numpy out;
CUDA tensors in -> CUDA tensors out.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from .. import _lib
from ..util import data as _data
from .Projector3DParallel import _device_of


class Line2DPlan:
    """Owns a vam_line2d_plan."""

    def __init__(self, n_y, n_x, angles_deg, det_count, device=None):
        self.device = _device_of(device)
        self.angles = np.ascontiguousarray(np.asarray(angles_deg, dtype=np.float64).ravel())
        self.shape_img = (int(n_y), int(n_x))
        self.shape_sino = (int(det_count), self.angles.size)
        h = ctypes.c_void_p()
        _lib.call("vam_line2d_plan_create", n_y, n_x, self.angles.size,
                  self.angles.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), det_count, self.device.index,
                  ctypes.byref(h))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.load().vam_line2d_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _run(self, name, x, in_shape, out_shape):
        x = torch.as_tensor(x, dtype=torch.float32, device=self.device).reshape(in_shape).contiguous()
        out = torch.empty(out_shape, dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.call(name, self._h, _lib.ptr(x), _lib.ptr(out), _lib.stream_ptr(torch.cuda.current_stream(self.device)))
        return out

    def forward(self, img):
        return self._run("vam_line2d_forward", img, self.shape_img, self.shape_sino)

    def backward(self, sino):
        return self._run("vam_line2d_backward", sino, self.shape_sino, self.shape_img)


class Projector2DParallelCUDAAstra:
    """ASTRA "line" model projector (Projector2DParallelCUDA.py:7-45): ``forward``
    clips its input to the inscribed circle in place; ``backward`` zeroes
    ``proj_geo.zero_dose_sino`` entries of its input in place, backprojects and clips."""

    def __init__(self, target_geo, proj_geo, device=None):
        self.target_geo = target_geo
        self.proj_geo = proj_geo
        arr = np.asarray(target_geo.array)
        self.nY, self.nX = arr.shape[:2]
        self.nT = self.nX
        self.angles = np.asarray(proj_geo.angles, dtype=np.float64)
        self.plan = Line2DPlan(self.nY, self.nX, self.angles, self.nT, device)
        self.device = self.plan.device
        self._inside = torch.as_tensor(_data.circle_inside_mask(self.nY, self.nX), device=self.device)

    def forward(self, target):
        """b = A x (Projector2DParallelCUDA.py:20-29)."""
        if isinstance(target, torch.Tensor):
            x = target.reshape(self.nY, self.nX)
            x[~self._inside.to(x.device)] = 0
            return self.plan.forward(x)
        x = _data.clipToCircle(np.asarray(target).reshape(self.nY, self.nX) if np.ndim(target) == 3 else target)
        return self.plan.forward(np.ascontiguousarray(x, dtype=np.float32)).double().cpu().numpy()

    def backward(self, sinogram):
        """x = A^T b (Projector2DParallelCUDA.py:31-45)."""
        b = sinogram
        zd = getattr(self.proj_geo, "zero_dose_sino", None)
        if zd is not None:
            b[torch.as_tensor(zd, device=b.device) if isinstance(b, torch.Tensor) else zd] = 0.0
        is_t = isinstance(b, torch.Tensor)
        x = self.plan.backward(b if is_t else np.ascontiguousarray(b, dtype=np.float32))
        x = x * self._inside
        return x if is_t else x.double().cpu().numpy()
