"""Parallel-beam projector on the B200: drop-in for the reference's projector family.

``Projector3DParallel`` implements the discretisation of
``Projector3DParallelPython`` (vamtoolbox/projector/Projector3DParallel.py:57-216):
rotate-and-sum forward with skimage-warp bilinear sampling (R1), pixel-driven
np.interp backprojection with the inscribed-circle clip (R2), and the
occlusion shadow of an attenuation field.  It also applies the radial
absorption mask that the reference's ASTRA classes apply
(Projector3DParallel.py:28-29, 51-52; Projector3DParallelCUDA.py:42-44, 66-67)
whenever ``proj_geo.absorption_coeff`` is set, so every parallel-beam dispatch
of ``projectorconstructor`` lands on one set of kernels.  ``adjoint`` is the
exact transpose of ``forward`` (the reference's backward is not).

Inputs may be numpy arrays (returned as float64 numpy, like the reference)
or CUDA torch tensors (float32, returned as CUDA tensors without a copy to
the host).
"""
from __future__ import annotations

import ctypes
import threading

import numpy as np
import torch

from .. import _lib

ABSORPTION_MODES = {None: _lib.ABS_NONE, "none": _lib.ABS_NONE, "mask": _lib.ABS_MASK, "ray": _lib.ABS_RAY}


def _device_of(device):
    if device is None:
        if not torch.cuda.is_available():
            raise RuntimeError("vamtoolbox_b200 projectors need a CUDA device (no CPU fallback)")
        return torch.device("cuda", torch.cuda.current_device())
    d = torch.device(device)
    if d.type != "cuda":
        raise RuntimeError("vamtoolbox_b200 projectors run on CUDA devices only")
    return d if d.index is not None else torch.device("cuda", torch.cuda.current_device())


# Idle plans of released ParallelPlan objects, by geometry: a plan (per-angle tables, the
# backprojection bin table, scratch volumes: hundreds of MB at 256^3) is kept when its last Python
# reference goes away and handed to the next ParallelPlan of the same shape, angles and device, reset
# to no absorption, no occlusion and the default launch shapes.  Repeated optimize() calls on one
# geometry then skip the device allocations and frees (cudaMalloc / cudaFree of the tables took
# 2-140 ms per plan, with the frees synchronising the device).  At most _POOL_MAX idle plans are kept
# (oldest destroyed first); clear_plan_pool() destroys them all.
_POOL_MAX = 4
_pool = []  # [(key, handle, has_backward_table)], oldest first
_pool_lock = threading.Lock()
_DEFAULT_TUNING = {"forward_vz": 0, "backward_vz": 0, "adjoint_vz": 0, "backward_batch": 2, "adjoint_table": 1,
                   "backward_table": 1, "forward_tma": 1}


def _pool_key(shape_vol, angles, device):
    return shape_vol, angles.tobytes(), str(device)


def _pool_take(key):
    with _pool_lock:
        for i, (k, h, tab) in enumerate(_pool):
            if k == key:
                del _pool[i]
                return h, tab
    return None


def _pool_give(key, h, tab):
    evicted = []
    with _pool_lock:
        _pool.append((key, h, tab))
        while len(_pool) > _POOL_MAX:
            evicted.append(_pool.pop(0)[1])
    for e in evicted:
        _lib.load().vam_parallel_plan_destroy(e)


def clear_plan_pool():
    """Destroy every idle plan kept for reuse (releases their device memory)."""
    with _pool_lock:
        items = list(_pool)
        _pool.clear()
    for _, h, _ in items:
        _lib.load().vam_parallel_plan_destroy(h)


class ParallelPlan:
    """Owns a vam_parallel_plan (per-angle tables, circle mask, occlusion, absorption).

    When the object is garbage collected its plan is kept for the next ParallelPlan of the same
    geometry (see ``clear_plan_pool``); ``close()`` destroys it instead."""

    def __init__(self, n_y, n_x, n_z, angles_deg, device=None):
        self.device = _device_of(device)
        self.shape_vol = (int(n_y), int(n_x), int(n_z))
        self.angles = np.ascontiguousarray(np.asarray(angles_deg, dtype=np.float64).ravel())
        self.shape_sino = (int(n_y), self.angles.size, int(n_z))
        self.absorption = None
        self.has_occlusion = False
        self._adj_ready = False
        # matched-transpose weight table: 16 B per pixel and angle (skipped above this size)
        self.adj_table_limit_bytes = 8 << 30
        # backprojection bin table (32 B per 2 x 2 pixel block inside the circle and angle, about 8 B per
        # pixel), built here for volumes of 64 slices and more, so it exists before any capture of a
        # backprojection
        self.bwd_table_limit_bytes = 8 << 30
        self.has_backward_table = False
        self._key = _pool_key(self.shape_vol, self.angles, self.device)
        reused = _pool_take(self._key)
        if reused is not None:
            self._h, self.has_backward_table = reused
            try:
                self._reset()
            except Exception:
                self.close()
                raise
            return
        geom = _lib.ParallelGeom(n_y, n_x, n_z, self.angles.size,
                                 self.angles.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self.device.index)
        h = ctypes.c_void_p()
        _lib.call("vam_parallel_plan_create", ctypes.byref(geom), ctypes.byref(h))
        self._h = h
        if int(n_z) % 4 == 0 and int(n_z) >= 64:
            self.prepare_backward()

    def _reset(self):
        """A reused plan: no absorption, no occlusion, the default launch shapes."""
        with torch.cuda.device(self.device):
            _lib.call("vam_parallel_set_absorption", self._h, _lib.ABS_NONE, None, 0.0, 1.0, self._stream())
            _lib.call("vam_parallel_clear_occlusion", self._h)
        self.set_tuning(dict(_DEFAULT_TUNING))

    @property
    def handle(self):
        return self._h

    def close(self):
        """Destroy the plan now (it is not kept for reuse)."""
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.load().vam_parallel_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            if getattr(self, "_h", None) is not None and self._h.value:
                h, self._h = self._h, None
                _pool_give(self._key, h, self.has_backward_table)
        except Exception:
            pass

    def _stream(self):
        return _lib.stream_ptr(torch.cuda.current_stream(self.device))

    def set_absorption(self, mode, mask=None, alpha_per_px=0.0, radius_px=1.0):
        code = ABSORPTION_MODES[mode]
        m = None
        if code == _lib.ABS_MASK:
            m = torch.as_tensor(np.ascontiguousarray(mask, dtype=np.float32), device=self.device)
            if tuple(m.shape) != self.shape_vol[:2]:
                raise ValueError(f"absorption mask must be {self.shape_vol[:2]}, got {tuple(m.shape)}")
        with torch.cuda.device(self.device):
            _lib.call("vam_parallel_set_absorption", self._h, code, _lib.ptr(m), float(alpha_per_px),
                      float(radius_px), self._stream())
            torch.cuda.current_stream(self.device).synchronize()
        self.absorption = mode
        self._adj_ready = False

    def prepare_adjoint(self):
        """Build the matched-transpose weight table (allocates; not during graph capture)."""
        nbytes = 16 * self.shape_vol[0] * self.shape_vol[1] * self.angles.size
        if nbytes > self.adj_table_limit_bytes:
            return False
        with torch.cuda.device(self.device):
            _lib.call("vam_parallel_prepare_adjoint", self._h, self._stream())
        self._adj_ready = True
        return True

    def prepare_backward(self):
        """Build the backprojection bin table (allocates; not during graph capture).  False when it would
        exceed ``bwd_table_limit_bytes``, the sinogram is too large for its 32-bit offsets or nZ % 4 != 0."""
        ny, nx, nz = self.shape_vol
        if (8 * ny * nx * (self.angles.size + 1) > self.bwd_table_limit_bytes or ny * self.angles.size * nz >= 2 ** 31
                or nz % 4 != 0):
            return False
        with torch.cuda.device(self.device):
            _lib.call("vam_parallel_prepare_backward", self._h, self._stream())
        self.has_backward_table = True
        return True

    _TUNING_FIELDS = ("forward_vz", "backward_vz", "adjoint_vz", "backward_batch", "adjoint_table", "backward_table",
                      "forward_tma")

    def set_tuning(self, tuning):
        """Set launch shapes: dict with any of forward_vz / backward_vz / adjoint_vz (0 auto, 1 generic,
        4, 8), backward_batch (1, 2, 4), adjoint_table, backward_table and forward_tma (0, 1); missing keys
        keep their value."""
        cur = self.get_tuning()
        unknown = set(tuning) - set(self._TUNING_FIELDS)
        if unknown:
            raise KeyError(f"unknown tuning fields {sorted(unknown)}")
        cur.update({k: int(v) for k, v in tuning.items()})
        t = _lib.ParallelTuning(*(cur[k] for k in self._TUNING_FIELDS))
        _lib.call("vam_parallel_set_tuning", self._h, ctypes.byref(t))

    def get_tuning(self):
        t = _lib.ParallelTuning()
        _lib.call("vam_parallel_get_tuning", self._h, ctypes.byref(t))
        return {k: int(getattr(t, k)) for k in self._TUNING_FIELDS}

    def autotune(self, use_cache=True, ops=("forward", "backward", "adjoint")):
        """Time the launch-shape candidates of ``ops`` on this plan's device (or reuse the cached winner)."""
        from ..autotune import autotune

        return autotune(self, use_cache=use_cache, ops=tuple(ops))

    def set_occlusion(self, insert):
        ins = torch.as_tensor(np.ascontiguousarray(np.atleast_3d(insert), dtype=np.float32), device=self.device)
        if tuple(ins.shape) != self.shape_vol:
            raise ValueError(f"attenuation field must be {self.shape_vol}, got {tuple(ins.shape)}")
        with torch.cuda.device(self.device):
            _lib.call("vam_parallel_set_occlusion", self._h, _lib.ptr(ins), self._stream())
            torch.cuda.current_stream(self.device).synchronize()
        self.has_occlusion = True

    def status(self):
        """Read and clear the plan's status bits (vam_status_bits; 0 = every launch completed its outputs).
        Synchronises the device."""
        v = ctypes.c_int32()
        with torch.cuda.device(self.device):
            _lib.call("vam_parallel_status", self._h, ctypes.byref(v))
        return int(v.value)

    def set_occlusion_2d(self, occlusion):
        """The 2-D class's digitised occlusion (Projector2DParallel.py:70-143) from a boolean [nY, nX]
        mask.  Raises ValueError where the reference's generateOccSinogram raises (an empty mask; occluded
        pixels both below the first detector bin and in the last bin at one angle)."""
        if self.shape_vol[2] != 1:
            raise ValueError("the digitised occlusion is defined for 2-D (single-slice) plans")
        occ = np.asarray(occlusion).reshape(-1)
        if occ.size != self.shape_vol[0] * self.shape_vol[1]:
            raise ValueError(f"occlusion must be {self.shape_vol[:2]}, got {np.shape(occlusion)}")
        m = torch.as_tensor(np.ascontiguousarray(occ != 0, dtype=np.uint8), device=self.device)
        with torch.cuda.device(self.device):
            try:
                _lib.call("vam_parallel_set_occlusion_2d", self._h, _lib.ptr(m), self._stream())
            except _lib.VamError as exc:
                if exc.code == _lib.VAM_ERR_SHAPE:
                    raise ValueError(exc.message) from exc
                raise
        self.has_occlusion = True

    def occlusion_sinogram_2d(self):
        """The float64 bin minima of the digitised 2-D occlusion, [nY, n_angles], NaN for empty bins."""
        out = torch.empty(self.shape_sino[:2], dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.call("vam_parallel_get_occlusion_sinogram_2d", self._h, _lib.ptr(out), self._stream())
        return out

    def occlusion_sinogram(self):
        out = torch.empty(self.shape_sino, dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.call("vam_parallel_get_occlusion_sinogram", self._h, _lib.ptr(out), self._stream())
        return out

    def _check(self, t, shape, name):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
            raise TypeError(f"{name}: expected a contiguous float32 CUDA tensor")
        if tuple(t.shape) != shape:
            raise ValueError(f"{name}: expected shape {shape}, got {tuple(t.shape)}")
        if t.device != self.device:
            raise ValueError(f"{name}: tensor on {t.device}, plan on {self.device}")

    def forward(self, vol, out=None):
        self._check(vol, self.shape_vol, "forward input")
        if out is None:
            out = torch.empty(self.shape_sino, dtype=torch.float32, device=self.device)
        self._check(out, self.shape_sino, "forward output")
        with torch.cuda.device(self.device):
            _lib.call("vam_parallel_forward", self._h, _lib.ptr(vol), _lib.ptr(out), self._stream())
        return out

    def backward_ref(self, sino, out=None):
        self._check(sino, self.shape_sino, "backward input")
        if out is None:
            out = torch.empty(self.shape_vol, dtype=torch.float32, device=self.device)
        self._check(out, self.shape_vol, "backward output")
        with torch.cuda.device(self.device):
            _lib.call("vam_parallel_backward_ref", self._h, _lib.ptr(sino), _lib.ptr(out), self._stream())
        return out

    def backward_ref_noclip(self, sino, out=None):
        """backward_ref without the inscribed-circle clip (Projector2DParallel.py:188, 230-231)."""
        self._check(sino, self.shape_sino, "backward input")
        if out is None:
            out = torch.empty(self.shape_vol, dtype=torch.float32, device=self.device)
        self._check(out, self.shape_vol, "backward output")
        with torch.cuda.device(self.device):
            _lib.call("vam_parallel_backward_ref_noclip", self._h, _lib.ptr(sino), _lib.ptr(out), self._stream())
        return out

    def adjoint(self, sino, out=None):
        self._check(sino, self.shape_sino, "adjoint input")
        if not self._adj_ready and not torch.cuda.is_current_stream_capturing():
            self.prepare_adjoint()
        if out is None:
            out = torch.empty(self.shape_vol, dtype=torch.float32, device=self.device)
        self._check(out, self.shape_vol, "adjoint output")
        with torch.cuda.device(self.device):
            _lib.call("vam_parallel_adjoint", self._h, _lib.ptr(sino), _lib.ptr(out), self._stream())
        return out


def _to_device(x, device, shape):
    """numpy / tensor -> contiguous float32 tensor on device with the given shape."""
    if isinstance(x, torch.Tensor):
        t = x.to(device=device, dtype=torch.float32)
    else:
        t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).to(device)
    t = t.reshape(shape).contiguous()
    return t


class Projector3DParallel:
    """B200 projector for ``projectorconstructor`` (parallel beam, nZ >= 1).

    Parameters
    ----------
    target_geo, proj_geo : geometry objects (vamtoolbox_b200.geometry or the reference's).
    absorption : None | "mask" | "ray"
        "mask" (default when ``proj_geo.absorption_coeff`` is set) applies the
        reference's radial mask; "ray" applies the per-sample exp(-a*(s-s_entry))
        weighting with a = absorption_coeff * projector_pixel_size (1/pixel) and
        the container radius in pixels.
    device : CUDA device (default: current).
    """

    def __init__(self, target_geo, proj_geo, absorption=None, device=None):
        self.target_geo = target_geo
        self.proj_geo = proj_geo
        arr = np.atleast_3d(target_geo.array)
        self.nY, self.nX, self.nZ = arr.shape
        self.angles = np.asarray(proj_geo.angles, dtype=np.float64)
        self.plan = ParallelPlan(self.nY, self.nX, self.nZ, self.angles, device)
        self.device = self.plan.device
        if absorption is None and getattr(proj_geo, "absorption_coeff", None) is not None:
            absorption = "mask"
        if absorption == "mask":
            mask = getattr(proj_geo, "absorption_mask", None)
            if mask is None:
                proj_geo.calcAbsorptionMask(target_geo)
                mask = proj_geo.absorption_mask
            mask = np.asarray(mask)
            self.plan.set_absorption("mask", mask=mask[:, :, 0] if mask.ndim == 3 else mask)
        elif absorption == "ray":
            px = proj_geo.projector_pixel_size
            self.plan.set_absorption("ray", alpha_per_px=float(proj_geo.absorption_coeff) * px,
                                     radius_px=float(proj_geo.container_radius) / px)
        self.absorption = absorption
        self._zd_src, self._zd_mask = None, None
        if getattr(proj_geo, "attenuation_field", None) is not None:
            att = np.atleast_3d(np.asarray(proj_geo.attenuation_field))
            self.plan.set_occlusion(np.where(att > 0, 1.0, 0.0))

    # -- zero-dose sinogram (geometry.ProjectionGeometry.calcZeroDoseSinogram) ----------------
    def _zero_dose_applies(self):
        # the reference's backward zeroes the entries in its ASTRA classes and 2-D classes
        # (Projector3DParallel.py:43-44, Projector3DParallelCUDA.py:57-58, Projector2DParallel.py:206-207),
        # not in the 3-D Python class it dispatches to when an attenuation field is set
        zd = getattr(self.proj_geo, "zero_dose_sino", None)
        return zd is not None and not (self.nZ > 1 and getattr(self.proj_geo, "attenuation_field", None) is not None)

    def zero_dose_mask(self):
        """The zero-dose entries as a device bool tensor of the sinogram's shape (built once per zero-dose
        array, so call it before any graph capture), or None when no zero-dose region applies."""
        if not self._zero_dose_applies():
            return None
        zd = self.proj_geo.zero_dose_sino
        if self._zd_src is not zd:
            self._zd_mask = torch.as_tensor(np.asarray(zd, dtype=bool), device=self.device).reshape(self.plan.shape_sino)
            self._zd_src = zd
        return self._zd_mask

    def zero_dose_(self, b):
        """b with its zero-dose entries set to 0 in place, as the reference's backward does before it
        projects (a numpy array or a device tensor; b itself is returned); nothing without a zero-dose
        region."""
        if not self._zero_dose_applies():
            return b
        if isinstance(b, torch.Tensor):
            m = self.zero_dose_mask()
            b.view(self.plan.shape_sino).masked_fill_(m if m.device == b.device else m.to(b.device), 0.0)
        else:
            b[np.asarray(self.proj_geo.zero_dose_sino, dtype=bool).reshape(np.shape(b))] = 0.0
        return b

    # -- device API ---------------------------------------------------------
    def forward_t(self, x, out=None):
        return self.plan.forward(_to_device(x, self.device, self.plan.shape_vol), out)

    def backward_t(self, b, out=None):
        return self.plan.backward_ref(self.zero_dose_(_to_device(b, self.device, self.plan.shape_sino)), out)

    def adjoint_t(self, b, out=None):
        return self.plan.adjoint(_to_device(b, self.device, self.plan.shape_sino), out)

    # -- reference API --------------------------------------------------------
    def forward(self, x):
        """Sinogram (nR, nA, nZ) of x (R1, Projector3DParallel.py:113-156)."""
        if isinstance(x, torch.Tensor) and x.is_cuda:
            return self.forward_t(x)
        return self.forward_t(x).double().cpu().numpy()

    def backward(self, b):
        """Reference-parity backprojection (R2, Projector3DParallel.py:158-207); the zero-dose entries of b
        are set to 0 in place first, as the reference's backward does."""
        self.zero_dose_(b)
        if isinstance(b, torch.Tensor) and b.is_cuda:
            return self.backward_t(b)
        return self.backward_t(b).double().cpu().numpy()

    def adjoint(self, b):
        """Exact transpose of forward."""
        if isinstance(b, torch.Tensor) and b.is_cuda:
            return self.adjoint_t(b)
        return self.adjoint_t(b).double().cpu().numpy()


# The reference's names for the same dispatch slots (projectorconstructor.py:74-160).  The
# ASTRA-model CUDA class (vector geometry, inclined rays) is projector/Projector3DParallelCUDA.py.
Projector3DParallelPython = Projector3DParallel
Projector3DParallelAstra = Projector3DParallel
