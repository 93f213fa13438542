"""Parallel beam in ASTRA's vector geometry: drop-in for the reference's
``Projector3DParallelCUDAAstra`` (vamtoolbox/projector/Projector3DParallelCUDA.py:13-72)
and ``genVectorsAstra`` (vamtoolbox/projector/genVectorsAstra.py:4-53).

The reference hands this geometry to ASTRA's CUDA projectors
(``create_sino3d_gpu`` / ``create_backprojection3d_gpu``); here it runs on
libvamcore's vector-geometry kernels (``vam_vec_*``): a Joseph-type forward
projector (every ray sampled on each voxel plane across its dominant axis,
bilinear within the plane, times |ray| / |ray_dominant|) and a voxel-driven
backprojector (bilinear on the detector).  It is the only projector of the
package for inclined rays (``proj_geo.inclination_angle``: laminography),
and is selected for parallel-beam geometries that set one, or with
``ProjectionGeometry(..., parallel_model="astra")``.  ASTRA is not available
to pin this model against; it follows ASTRA's published geometry
conventions (volume centred on the origin, detector pixel (0, 0) at
d - (nU/2 - 1/2) u - (nV/2 - 1/2) v) and interpolates with full float32
weights where ASTRA's texture units use 8-bit fractions.

Array layouts are the reference's after its transposes: target [nY][nX][nZ],
sinogram [nT = nX][nA][nZ].  numpy in -> float64 numpy out; CUDA tensors in
-> CUDA tensors out.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from .. import _lib
from ..util import data as _data
from .Projector3DParallel import _device_of, _to_device


def genVectorsAstra(angles, incline_angle, cone_angle=0, distance_origin_source=0):
    """ASTRA ``parallel3d_vec`` rows for rays inclined by ``incline_angle`` degrees
    (genVectorsAstra.py:4-53): ray (sin a, -cos a, sin i), detector centre 0,
    u = (cos a, sin a, 0), v = (sin a cos i, -cos a cos i, cos i).  With a
    non-zero ``cone_angle`` the rows hold the reference's cone variant (source,
    detector centre at +-``distance_origin_source``), which no projector of the
    reference consumes."""
    angles = np.deg2rad(np.atleast_1d(np.asarray(angles, dtype=np.float64)))
    inc = np.deg2rad(incline_angle)
    vec = np.zeros((angles.size, 12))
    s, c = np.sin(angles), np.cos(angles)
    if cone_angle == 0:
        vec[:, 0], vec[:, 1], vec[:, 2] = s, -c, np.sin(inc)
    else:
        D = distance_origin_source
        vec[:, 0], vec[:, 1], vec[:, 2] = s * D, -c * D, np.sin(inc) * D
        vec[:, 3], vec[:, 4], vec[:, 5] = -s * D, c * D, -np.sin(inc) * D
    vec[:, 6], vec[:, 7], vec[:, 8] = c, s, 0
    vec[:, 9], vec[:, 10], vec[:, 11] = s * np.cos(inc), -c * np.cos(inc), np.cos(inc)
    return vec


def parallel3d_vectors(angles_rad, det_spacing_x=1.0, det_spacing_y=1.0):
    """ASTRA's ``parallel3d`` geometry as vector rows: ray (sin a, -cos a, 0),
    detector centre 0, u = (cos a, sin a, 0) * det_spacing_x, v = (0, 0, det_spacing_y)."""
    a = np.atleast_1d(np.asarray(angles_rad, dtype=np.float64))
    vec = np.zeros((a.size, 12))
    vec[:, 0], vec[:, 1] = np.sin(a), -np.cos(a)
    vec[:, 6], vec[:, 7] = np.cos(a) * det_spacing_x, np.sin(a) * det_spacing_x
    vec[:, 11] = det_spacing_y
    return vec


class VecPlan:
    """Owns a vam_vec_plan: volume [nY][nX][nZ], detector nU x nV, vector rows."""

    def __init__(self, n_y, n_x, n_z, vectors, det_cols, det_rows, device=None):
        self.device = _device_of(device)
        self.vectors = np.ascontiguousarray(np.asarray(vectors, dtype=np.float64).reshape(-1, 12))
        self.shape_vol = (int(n_y), int(n_x), int(n_z))
        self.shape_sino = (int(det_cols), self.vectors.shape[0], int(det_rows))
        geom = _lib.VecGeom(n_y, n_x, n_z, self.vectors.shape[0], det_cols, det_rows,
                            self.vectors.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self.device.index)
        h = ctypes.c_void_p()
        _lib.call("vam_vec_plan_create", ctypes.byref(geom), ctypes.byref(h))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.load().vam_vec_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        f, b = ctypes.c_int32(), ctypes.c_int32()
        _lib.call("vam_vec_plan_info", self._h, ctypes.byref(f), ctypes.byref(b))
        return {"flat_forward": bool(f.value), "flat_backward": bool(b.value)}

    def _check(self, t, shape, name):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
            raise TypeError(f"{name}: expected a contiguous float32 CUDA tensor")
        if tuple(t.shape) != shape or t.device != self.device:
            raise ValueError(f"{name}: expected shape {shape} on {self.device}, got {tuple(t.shape)} on {t.device}")

    def forward(self, vol, out=None):
        self._check(vol, self.shape_vol, "forward input")
        out = torch.empty(self.shape_sino, dtype=torch.float32, device=self.device) if out is None else out
        self._check(out, self.shape_sino, "forward output")
        with torch.cuda.device(self.device):
            _lib.call("vam_vec_forward", self._h, _lib.ptr(vol), _lib.ptr(out),
                      _lib.stream_ptr(torch.cuda.current_stream(self.device)))
        return out

    def adjoint(self, sino, out=None):
        """Exact transpose of ``forward`` (float atomics; for gradients)."""
        self._check(sino, self.shape_sino, "adjoint input")
        out = torch.empty(self.shape_vol, dtype=torch.float32, device=self.device) if out is None else out
        self._check(out, self.shape_vol, "adjoint output")
        with torch.cuda.device(self.device):
            _lib.call("vam_vec_adjoint", self._h, _lib.ptr(sino), _lib.ptr(out),
                      _lib.stream_ptr(torch.cuda.current_stream(self.device)))
        return out

    def backward(self, sino, out=None):
        self._check(sino, self.shape_sino, "backward input")
        out = torch.empty(self.shape_vol, dtype=torch.float32, device=self.device) if out is None else out
        self._check(out, self.shape_vol, "backward output")
        with torch.cuda.device(self.device):
            _lib.call("vam_vec_backward", self._h, _lib.ptr(sino), _lib.ptr(out),
                      _lib.stream_ptr(torch.cuda.current_stream(self.device)))
        return out


class Projector3DParallelCUDAAstra:
    """ASTRA-model parallel-beam projector (Projector3DParallelCUDA.py:13-72).

    ``forward`` clips its input to the inscribed circle in place and applies
    the absorption mask first (:40-54); ``backward`` zeroes
    ``proj_geo.zero_dose_sino`` entries of its input in place, backprojects,
    applies the mask and clips (:56-72).  The reference also transposes
    ``proj_geo.absorption_mask`` in place for ASTRA's axis order; this class
    works in the reference's own [nY][nX][nZ] order and leaves it as it is.
    """

    def __init__(self, target_geo, proj_geo, device=None):
        self.target_geo = target_geo
        self.proj_geo = proj_geo
        arr = np.atleast_3d(np.asarray(target_geo.array))
        self.nY, self.nX, self.nZ = arr.shape
        self.nT = self.nX
        self.angles_rad = np.deg2rad(np.asarray(proj_geo.angles, dtype=np.float64))
        incl = getattr(proj_geo, "inclination_angle", None)
        if incl is None or incl == 0:
            self.vectors = parallel3d_vectors(self.angles_rad)
        else:
            self.vectors = genVectorsAstra(proj_geo.angles, incl)
        self.plan = VecPlan(self.nY, self.nX, self.nZ, self.vectors, self.nT, self.nZ, device)
        self.device = self.plan.device
        self._mask = None
        if getattr(proj_geo, "absorption_coeff", None) is not None:
            if getattr(proj_geo, "absorption_mask", None) is None:
                proj_geo.calcAbsorptionMask(target_geo)
            m = np.asarray(proj_geo.absorption_mask, dtype=np.float32)
            m = m if m.ndim == 3 else m[:, :, None]
            self._mask = torch.from_numpy(np.ascontiguousarray(np.broadcast_to(m, (self.nY, self.nX, self.nZ)))
                                          ).to(self.device)
        self._circle = torch.from_numpy(_data.circle_inside_mask(self.nY, self.nX).astype(np.float32)).to(
            self.device)[:, :, None]

    # -- device API ---------------------------------------------------------
    def forward_t(self, x, out=None):
        x = _to_device(x, self.device, self.plan.shape_vol) * self._circle
        if self._mask is not None:
            x = x * self._mask
        return self.plan.forward(x.contiguous(), out)

    def backward_t(self, b, out=None):
        vol = self.plan.backward(_to_device(b, self.device, self.plan.shape_sino), out)
        if self._mask is not None:
            vol.mul_(self._mask)
        return vol.mul_(self._circle)

    # -- reference API --------------------------------------------------------
    def forward(self, target):
        """b = A x (Projector3DParallelCUDA.py:40-54); the input is clipped in place."""
        if isinstance(target, np.ndarray):
            _data.clipToCircle(target)
            return self.forward_t(target).double().cpu().numpy()
        return self.forward_t(target)

    def backward(self, sinogram):
        """x = A^T b (Projector3DParallelCUDA.py:56-72); zero-dose entries of the input are zeroed in place."""
        zd = getattr(self.proj_geo, "zero_dose_sino", None)
        if zd is not None:
            if isinstance(sinogram, torch.Tensor):
                sinogram[torch.as_tensor(zd, device=sinogram.device)] = 0.0
            else:
                sinogram[zd] = 0.0
        if isinstance(sinogram, torch.Tensor) and sinogram.is_cuda:
            return self.backward_t(sinogram)
        return self.backward_t(sinogram).double().cpu().numpy()
