"""ctypes binding of libvamcore.so (include/vam.h).

The library is built in-tree by ``vamtoolbox_b200.csrc.build`` and loaded
from the package directory.  There is no fallback: if the library is missing
or a call fails, a RuntimeError carrying the C status and message is raised.
"""
from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libvamcore.so"

VAM_OK, VAM_ERR_ARG, VAM_ERR_SHAPE, VAM_ERR_CUDA, VAM_ERR_TIMEOUT, VAM_ERR_NOTSUP, VAM_ERR_NOMEM = range(7)
_STATUS = {0: "VAM_OK", 1: "VAM_ERR_ARG", 2: "VAM_ERR_SHAPE", 3: "VAM_ERR_CUDA", 4: "VAM_ERR_TIMEOUT",
           5: "VAM_ERR_NOTSUP", 6: "VAM_ERR_NOMEM"}

ABS_NONE, ABS_MASK, ABS_RAY = 0, 1, 2
RED_MAX, RED_MIN, RED_SUM = 0, 1, 2
PARAM = {"physical_path_length": 0, "canonical": 1, "optical_path_length": 2}
SOLVER = {"forward_symplectic_euler": 0, "forward_euler": 1, "leapfrog": 2}
INDEX_HOMOGENEOUS, INDEX_GRID, INDEX_LUNEBURG = 0, 1, 2
ALPHA_ZERO, ALPHA_CYLINDER, ALPHA_BALL, ALPHA_GRID = 0, 1, 2, 3

_c_int = ctypes.c_int
_c_i32 = ctypes.c_int32
_c_i64 = ctypes.c_int64
_c_f = ctypes.c_float
_c_d = ctypes.c_double
_vp = ctypes.c_void_p


class VamError(RuntimeError):
    def __init__(self, func, code, msg):
        super().__init__(f"{func} failed with {_STATUS.get(code, code)}: {msg}")
        self.code = code
        self.message = msg


class ParallelGeom(ctypes.Structure):
    _fields_ = [("n_y", _c_i32), ("n_x", _c_i32), ("n_z", _c_i32), ("n_angles", _c_i32),
                ("angles_deg", ctypes.POINTER(_c_d)), ("device", _c_i32)]


class RayGeom(ctypes.Structure):
    _fields_ = [("n_x", _c_i32), ("n_y", _c_i32), ("n_z", _c_i32),
                ("coord_min", _c_d * 3), ("coord_max", _c_d * 3), ("voxel", _c_d * 3),
                ("step_size", _c_d), ("max_num_step", _c_i32), ("num_step_per_exit_check", _c_i32),
                ("parametrization", _c_i32), ("ode_solver", _c_i32), ("num_rays", _c_i64), ("device", _c_i32)]


class RayMedium(ctypes.Structure):
    _fields_ = [("index_kind", _c_i32), ("n_sur", _c_f), ("lune_R", _c_f), ("lune_p", _c_f),
                ("n_grid_dev", _vp), ("grad_n_grid_dev", _vp),
                ("atten_kind", _c_i32), ("atten_value", _c_f), ("atten_R", _c_f), ("atten_grid_dev", _vp),
                ("absorb_at_grid_dev", _vp)]


class ParallelTuning(ctypes.Structure):
    _fields_ = [("forward_vz", _c_i32), ("backward_vz", _c_i32), ("adjoint_vz", _c_i32),
                ("backward_batch", _c_i32), ("adjoint_table", _c_i32), ("backward_table", _c_i32),
                ("forward_tma", _c_i32)]


OP_FORWARD, OP_BACKWARD_REF, OP_ADJOINT = 0, 1, 2


class Work(ctypes.Structure):
    _fields_ = [("plan", _vp), ("op", _c_i32), ("in_", _vp), ("out", _vp)]


class BclpParams(ctypes.Structure):
    _fields_ = [("table_f", _vp), ("table_map", _vp), ("table_dmap", _vp), ("n_table", _c_i32),
                ("table_f0", _c_f), ("table_inv_step", _c_f),
                ("eps", _c_f), ("weight", _c_f), ("p", _c_f), ("eps_dev", _vp), ("weight_dev", _vp),
                ("response", _c_i32), ("resp_A", _c_d), ("resp_K", _c_d), ("resp_B", _c_d), ("resp_M", _c_d),
                ("resp_nu", _c_d), ("resp_C", _c_d)]


RESP_TABLE, RESP_GLF, RESP_LINEAR, RESP_IDENTITY = 0, 1, 2, 3


# name -> (argtypes, restype)
class VecGeom(ctypes.Structure):
    _fields_ = [("n_y", _c_i32), ("n_x", _c_i32), ("n_z", _c_i32), ("n_angles", _c_i32),
                ("det_cols", _c_i32), ("det_rows", _c_i32), ("vectors", ctypes.POINTER(_c_d)), ("device", _c_i32)]


class FrameParams(ctypes.Structure):
    _fields_ = [("n_u", _c_i32), ("n_v", _c_i32), ("src_col_dev", _vp), ("src_row_dev", _vp),
                ("bit_depth", _c_i32), ("has_norm", _c_i32), ("norm_value", _c_d), ("norm_dtype", _c_i32),
                ("has_scale", _c_i32), ("intensity_scale", _c_d), ("scale_is_f64", _c_i32),
                ("box_v0", _c_i32), ("box_v1", _c_i32), ("box_u0", _c_i32), ("box_u1", _c_i32)]


DTYPE_F32, DTYPE_F64 = 0, 1


_SIGS = {
    "vam_last_error_string": ([], ctypes.c_char_p),
    "vam_version": ([], ctypes.c_char_p),
    "vam_parallel_plan_create": ([ctypes.POINTER(ParallelGeom), ctypes.POINTER(_vp)], _c_int),
    "vam_parallel_plan_destroy": ([_vp], _c_int),
    "vam_parallel_set_absorption": ([_vp, _c_int, _vp, _c_f, _c_f, _vp], _c_int),
    "vam_parallel_set_occlusion": ([_vp, _vp, _vp], _c_int),
    "vam_parallel_set_occlusion_2d": ([_vp, _vp, _vp], _c_int),
    "vam_parallel_get_occlusion_sinogram_2d": ([_vp, _vp, _vp], _c_int),
    "vam_parallel_clear_occlusion": ([_vp], _c_int),
    "vam_parallel_get_occlusion_sinogram": ([_vp, _vp, _vp], _c_int),
    "vam_parallel_forward": ([_vp, _vp, _vp, _vp], _c_int),
    "vam_parallel_backward_ref": ([_vp, _vp, _vp, _vp], _c_int),
    "vam_parallel_backward_ref_noclip": ([_vp, _vp, _vp, _vp], _c_int),
    "vam_parallel_adjoint": ([_vp, _vp, _vp, _vp], _c_int),
    "vam_parallel_prepare_adjoint": ([_vp, _vp], _c_int),
    "vam_parallel_prepare_backward": ([_vp, _vp], _c_int),
    "vam_parallel_status": ([_vp, ctypes.POINTER(_c_i32)], _c_int),
    "vam_parallel_set_tuning": ([_vp, ctypes.POINTER(ParallelTuning)], _c_int),
    "vam_parallel_get_tuning": ([_vp, ctypes.POINTER(ParallelTuning)], _c_int),
    "vam_ray_record_count": ([_vp, _vp, _vp], _c_int),
    "vam_ray_record_fill": ([_vp, _vp, _vp, _vp, _vp], _c_int),
    "vam_csr_spmm": ([ctypes.c_int64, _vp, _vp, _vp, _vp, _c_i32, _vp, _vp], _c_int),
    "vam_batch_create": ([_c_i32, ctypes.POINTER(_vp)], _c_int),
    "vam_batch_destroy": ([_vp], _c_int),
    "vam_batch_submit": ([_vp, ctypes.POINTER(Work), _c_i32, _vp], _c_int),
    "vam_batch_prepare": ([_vp, ctypes.POINTER(Work), _c_i32, _vp], _c_int),
    "vam_batch_info": ([_vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(_c_i32)], _c_int),
    "vam_ray_plan_create": ([ctypes.POINTER(RayGeom), _vp, _vp, _c_f, ctypes.POINTER(_vp)], _c_int),
    "vam_ray_plan_destroy": ([_vp], _c_int),
    "vam_ray_set_medium": ([_vp, ctypes.POINTER(RayMedium), _vp], _c_int),
    "vam_ray_integrate": ([_vp, _vp, _vp, _vp], _c_int),
    "vam_ray_deposit": ([_vp, _vp, _vp, _vp], _c_int),
    "vam_ray_grad_alpha": ([_vp, _vp, _vp, _vp, _vp, _vp], _c_int),
    "vam_ray_active_at_cap": ([_vp, ctypes.POINTER(_c_i64)], _c_int),
    "vam_ray_prepare_trajectories": ([_vp, _c_i64, _vp], _c_int),
    "vam_ray_drop_trajectories": ([_vp], _c_int),
    "vam_reduce_workspace_bytes": ([_c_i64], ctypes.c_size_t),
    "vam_reduce": ([_vp, _c_i64, _c_int, _vp, _vp, ctypes.c_size_t, _vp], _c_int),
    "vam_reduce_noalloc": ([_vp, _c_i64, _c_int, _vp, _vp], _c_int),
    "vam_metric_ver": ([_vp, _vp, _c_i64, _vp, _vp, ctypes.c_size_t, _vp], _c_int),
    "vam_metric_ipdr": ([_vp, _vp, _c_i64, _vp, _vp, ctypes.c_size_t, _vp], _c_int),
    "vam_spectrum_scale": ([_vp, _vp, _c_i64, _c_i64, _vp], _c_int),
    "vam_filter_epilogue": ([_vp, _c_i64, _c_i64, _c_d, _c_int, _c_d, _c_int, _c_d, _vp, _vp], _c_int),
    "vam_bclp_dose_pass": ([_vp, _vp, _c_i64, ctypes.POINTER(BclpParams), _vp, _vp, _vp, _vp, ctypes.c_size_t, _vp],
                           _c_int),
    "vam_bclp_sino_update": ([_vp, _vp, _c_i64, _c_f, _c_f, _c_f, _c_f, _c_f, _c_int, _vp, _vp], _c_int),
    "vam_cal_threshold": ([_vp, _vp, _vp, _c_i64, _c_f, _c_f, _vp, _vp], _c_int),
    "vam_cal_sino_update": ([_vp, _vp, _vp, _c_i64, _c_f, _c_f, _c_i32, _vp], _c_int),
    "vam_scale_by_device": ([_vp, _vp, _c_i64, _c_int, _c_f, _vp], _c_int),
    "vam_osmo_model_update": ([_vp, _vp, _vp, _vp, _c_i64, _c_int, _c_f, _vp], _c_int),
    "vam_append": ([_vp, _c_i32, _vp, _vp, _c_i32, _vp], _c_int),
    "vam_vec_plan_create": ([ctypes.POINTER(VecGeom), ctypes.POINTER(_vp)], _c_int),
    "vam_vec_plan_destroy": ([_vp], _c_int),
    "vam_vec_plan_info": ([_vp, ctypes.POINTER(_c_i32), ctypes.POINTER(_c_i32)], _c_int),
    "vam_vec_forward": ([_vp, _vp, _vp, _vp], _c_int),
    "vam_vec_backward": ([_vp, _vp, _vp, _vp], _c_int),
    "vam_vec_adjoint": ([_vp, _vp, _vp, _vp], _c_int),
    "vam_line2d_plan_create": ([_c_i32, _c_i32, _c_i32, ctypes.POINTER(_c_d), _c_i32, _c_i32, ctypes.POINTER(_vp)],
                               _c_int),
    "vam_line2d_plan_destroy": ([_vp], _c_int),
    "vam_line2d_forward": ([_vp, _vp, _vp, _vp], _c_int),
    "vam_line2d_backward": ([_vp, _vp, _vp, _vp], _c_int),
    "vam_sino_rotate": ([_vp, _c_int, _c_i32, _c_i32, _c_i32, _c_i32, _c_i32, ctypes.POINTER(_c_d), _vp, _c_i32,
                         _c_i32, _vp], _c_int),
    "vam_sino_resize": ([_vp, _c_int, _c_i32, _c_i32, _c_i32, _c_i32, _c_i32, _vp, _c_i32, _c_i32, _vp], _c_int),
    "vam_select_workspace_bytes": ([], ctypes.c_size_t),
    "vam_select_pair": ([_vp, _c_int, _c_i64, _c_i64, _c_i64, _vp, _vp, ctypes.c_size_t, _vp], _c_int),
    "vam_imageseq_frames": ([_vp, _c_int, _c_i32, _c_i32, _c_i32, ctypes.POINTER(FrameParams), _vp, _vp], _c_int),
    "vam_rebin_fan": ([_vp, _c_int, _c_i32, _c_i32, _c_i32, _c_i32, _c_i32, _vp, _vp, _vp, _vp, _vp, _vp], _c_int),
}

_lib = None
_lock = threading.Lock()


def exported_symbols():
    return sorted(_SIGS)


def load() -> ctypes.CDLL:
    """Load libvamcore.so (raises if it was never built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m vamtoolbox_b200.csrc.build` "
                "(there is no CPU fallback for the projection kernels)")
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (args, res) in _SIGS.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib


def call(name, *args):
    lib = load()
    code = getattr(lib, name)(*args)
    if code != VAM_OK:
        msg = lib.vam_last_error_string().decode(errors="replace")
        raise VamError(name, code, msg)
    return code


def version() -> str:
    return load().vam_version().decode()


def ptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
