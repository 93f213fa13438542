"""CPU parity oracle for the VAMToolbox projection hot path.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by bench.py's CPU-baseline / reference legs, always as the checker or the
timed CPU baseline, never by the product package ``vamtoolbox_b200``.

It wraps ``oracle/vamoracle.c`` (float64 restatement of
vamtoolbox/projector/Projector3DParallel.py:77-216 and of the ray tracer
vamtoolbox/projector/pyTorchRayTrace.py:378-571, 738-775, 835-1143,
1253-1424) through ctypes, plus small numpy restatements of the optimizer
helpers (vamtoolbox/util/data.py, vamtoolbox/response.py,
vamtoolbox/metrics.py) used to check the fused device iteration bodies.
The library is pinned against golden vectors produced by the reference's
own code (tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_SRC = _HERE / "vamoracle.c"
_LIB = _HERE / "_build" / "libvamoracle.so"

_lib = None


def build(force: bool = False) -> Path:
    """Compile vamoracle.c with gcc (-O2 -fopenmp -ffp-contract=off)."""
    if _LIB.exists() and not force and _LIB.stat().st_mtime >= _SRC.stat().st_mtime:
        return _LIB
    _LIB.parent.mkdir(parents=True, exist_ok=True)
    cmd = [
        "gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC",
        "-o", str(_LIB), str(_SRC), "-lm",
    ]
    subprocess.run(cmd, check=True)
    return _LIB


def _load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(_LIB))
        dp = ctypes.POINTER(ctypes.c_double)
        u8p = ctypes.POINTER(ctypes.c_uint8)
        fp = ctypes.POINTER(ctypes.c_float)
        i = ctypes.c_int
        d = ctypes.c_double
        lib.orc_parallel_forward.argtypes = [dp, i, i, i, dp, i, dp, u8p, i, dp, d, d, dp]
        lib.orc_parallel_adjoint.argtypes = [dp, i, i, i, dp, i, dp, u8p, i, dp, d, d, dp]
        lib.orc_parallel_backward_ref.argtypes = [dp, i, i, i, dp, i, dp, i, dp, d, d, dp]
        lib.orc_occlusion_sinogram.argtypes = [dp, i, i, i, dp, i, dp, u8p]
        lib.orc_ray_trace.argtypes = [ctypes.c_void_p, fp, fp, ctypes.c_float, ctypes.c_long, i, dp, fp, fp, dp]
        lib.orc_ray_trace.restype = ctypes.c_long
        lib.orc_num_threads.restype = i
        lib.orc_set_num_threads.argtypes = [i]
        _lib = lib
    return _lib


def _p(a, ct=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(ct)) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def num_threads() -> int:
    return _load().orc_num_threads()


def set_num_threads(n: int) -> None:
    _load().orc_set_num_threads(int(n))


# --------------------------------------------------------------------------
# parallel beam
# --------------------------------------------------------------------------

def _abs_args(absorption):
    """absorption: None | ("mask", mask[nY,nX]) | ("ray", alpha_per_px, radius_px)."""
    if absorption is None:
        return 0, None, 0.0, 0.0
    if absorption[0] == "mask":
        return 1, _f64(absorption[1]), 0.0, 0.0
    if absorption[0] == "ray":
        return 2, None, float(absorption[1]), float(absorption[2])
    raise ValueError(absorption)


def occlusion_sinogram(insert, angles_deg):
    x = _f64(np.atleast_3d(insert))
    nY, nX, nZ = x.shape
    ang = _f64(angles_deg)
    occ = np.empty((nY, ang.size, nZ))
    flag = np.empty((ang.size, nZ), dtype=np.uint8)
    _load().orc_occlusion_sinogram(_p(x), nY, nX, nZ, _p(ang), ang.size, _p(occ), _p(flag, ctypes.c_uint8))
    return occ, flag


def parallel_forward(x, angles_deg, occlusion=None, absorption=None):
    """R1: Projector3DParallelPython.forward, float64.  occlusion = (occ, flag)."""
    x = _f64(np.atleast_3d(x))
    nY, nX, nZ = x.shape
    ang = _f64(angles_deg)
    b = np.empty((nY, ang.size, nZ))
    occ, flag = (None, None) if occlusion is None else (_f64(occlusion[0]), np.ascontiguousarray(occlusion[1], np.uint8))
    mode, mask, alpha, R = _abs_args(absorption)
    _load().orc_parallel_forward(_p(x), nY, nX, nZ, _p(ang), ang.size, _p(occ), _p(flag, ctypes.c_uint8),
                                 mode, _p(mask), alpha, R, _p(b))
    return b


def parallel_adjoint(b, angles_deg, occlusion=None, absorption=None):
    """Exact transpose of parallel_forward (float64, scatter form)."""
    b = _f64(b)
    nY, nA, nZ = b.shape
    ang = _f64(angles_deg)
    x = np.empty((nY, nY, nZ))
    occ, flag = (None, None) if occlusion is None else (_f64(occlusion[0]), np.ascontiguousarray(occlusion[1], np.uint8))
    mode, mask, alpha, R = _abs_args(absorption)
    _load().orc_parallel_adjoint(_p(b), nY, nY, nZ, _p(ang), nA, _p(occ), _p(flag, ctypes.c_uint8),
                                 mode, _p(mask), alpha, R, _p(x))
    return x


def parallel_backward_ref(b, angles_deg, occlusion=None, absorption=None):
    """R2: Projector3DParallelPython.backward (np.interp + clipToCircle), float64."""
    b = _f64(b)
    nY, nA, nZ = b.shape
    ang = _f64(angles_deg)
    x = np.empty((nY, nY, nZ))
    occ = None if occlusion is None else _f64(occlusion[0])
    mode, mask, alpha, R = _abs_args(absorption)
    _load().orc_parallel_backward_ref(_p(b), nY, nY, nZ, _p(ang), nA, _p(occ), mode, _p(mask), alpha, R, _p(x))
    return x


def occlusion_sinogram_2d(occlusion, angles_deg):
    """Projector2DParallelPython.generateOccSinogram (vamtoolbox/projector/Projector2DParallel.py:70-143):
    per angle, the pixels' detector coordinate t = x cos - y sin is binned with np.digitize over the
    sorted detector axis (a coordinate below the first bin index -1, i.e. the last bin's value), and
    each bin holding occluded pixels gets the least s = x sin + y cos among them; other bins are NaN.
    The values are assigned to the sorted unique bin indices in ascending order of the bins' values,
    as the reference's np.split / np.unique steps do.  occlusion: boolean [n, n].  Returns [n, nA]."""
    occ = np.asarray(occlusion, dtype=bool)
    n = occ.shape[0]
    C = n // 2
    y, x = np.mgrid[:n, :n] - C
    proj_t = np.arange(n) - C
    ang = np.deg2rad(np.asarray(angles_deg, dtype=np.float64))
    out = np.zeros((n, ang.size))
    bins = np.sort(proj_t)
    for i, a in enumerate(ang):
        c, s_ = np.cos(a), np.sin(a)
        t = x * c - y * s_
        s = x * s_ + y * c
        k = np.digitize(t, bins=bins) - 1
        td = proj_t[k]
        t_occ, s_occ = td[occ], s[occ]
        order = np.argsort(t_occ)  # any order within a bin: only each bin's minimum is kept
        t_sorted, s_sorted = t_occ[order], s_occ[order]
        starts = np.unique(t_sorted, return_index=True)[1]
        mins = [np.min(g) for g in np.split(s_sorted, starts[1:])] if t_sorted.size else []
        col = np.full(n, np.nan)
        col[np.unique(k[occ])] = mins
        out[:, i] = col
    return out


def parallel_forward_2d_occluded(x, angles_deg, occ_sinogram):
    """Projector2DParallelPython.forward with an occlusion (Projector2DParallel.py:145-186): the input
    clipped to the circle, rotated, samples with y > occ[j] (the detector column's least occluded s)
    zeroed, columns summed.  The same shadow rule as the 3-D forward, applied at every angle."""
    occ = _f64(occ_sinogram)[:, :, None]
    flag = np.ones((occ.shape[1], 1), dtype=np.uint8)
    return parallel_forward(clip_to_circle(x)[:, :, None], angles_deg, occlusion=(occ, flag))[:, :, 0]


def parallel_backward_2d_occluded(b, angles_deg, occ_sinogram, clipping=True):
    """Projector2DParallelPython.backward with an occlusion (Projector2DParallel.py:188-233 and its
    getOccShadow :240-247): per angle np.interp of the projection at t (left = right = 0), zeroed where
    s exceeds the occlusion value of t's np.digitize bin (no shadow where that value is NaN), summed
    over angles and, with clipping, clipped to the circle (the reference clips after every angle, which
    equals one clip at the end)."""
    b = _f64(b)
    n, na = b.shape
    C = n // 2
    y, x = np.mgrid[:n, :n] - C
    proj_t = np.arange(n) - C
    bins = np.sort(proj_t)
    occ = _f64(occ_sinogram)
    out = np.zeros((n, n))
    for i, a in enumerate(np.deg2rad(np.asarray(angles_deg, dtype=np.float64))):
        c, s_ = np.cos(a), np.sin(a)
        t = x * c - y * s_
        s = x * s_ + y * c
        back = np.interp(t, proj_t, b[:, i], left=0, right=0)
        td = proj_t[np.digitize(t, bins=bins) - 1]
        with np.errstate(invalid="ignore"):
            shadow = s > np.interp(td, proj_t, occ[:, i], left=np.nan, right=np.nan)
        out += back * np.logical_not(shadow)
    return clip_to_circle(out) if clipping else out


# --------------------------------------------------------------------------
# ray tracer
# --------------------------------------------------------------------------

class _RayCfg(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("span", ctypes.c_double * 3), ("xmax", ctypes.c_double * 3), ("xmin", ctypes.c_double * 3),
        ("voxel", ctypes.c_double * 3), ("norm", ctypes.c_double * 3),
        ("h32", ctypes.c_float), ("h_idx", ctypes.c_double),
        ("max_steps", ctypes.c_int), ("check_every", ctypes.c_int), ("twod", ctypes.c_int),
        ("n_kind", ctypes.c_int), ("n_sur", ctypes.c_float),
        ("n_grid", ctypes.POINTER(ctypes.c_double)), ("g_grid", ctypes.POINTER(ctypes.c_double)),
        ("a_kind", ctypes.c_int), ("a_val", ctypes.c_float), ("a_R", ctypes.c_float),
        ("a_grid", ctypes.POINTER(ctypes.c_double)), ("absorb", ctypes.POINTER(ctypes.c_double)),
    ]


def central_difference(n, voxel):
    """medium.py:224-273: central differences, zero boundary faces, none in 2D z."""
    n = np.asarray(n, dtype=np.float64)
    g = np.zeros(n.shape + (3,))
    g[1:-1, :, :, 0] = (n[2:] - n[:-2]) / (2 * voxel[0])
    g[:, 1:-1, :, 1] = (n[:, 2:] - n[:, :-2]) / (2 * voxel[1])
    if n.shape[2] > 1 and np.isfinite(voxel[2]):
        g[:, :, 1:-1, 2] = (n[:, :, 2:] - n[:, :, :-2]) / (2 * voxel[2])
    return g


def ray_trace(mode, grid, x0, v0, energy0=1.0, f=None, g=None, *, step_size, max_num_step,
              n_kind=0, n_sur=1.0, n_grid=None, grad_grid=None, a_kind=0, a_val=0.0, a_R=0.0,
              a_grid=None, absorb=None, check_every=10):
    """Trace rays like PyTorchRayTracingPropagator (symplectic Euler, physical path).

    grid: dict with xv, yv, zv coordinate vectors (float64).  mode "integrate"
    returns (g[nrays] float32, active_at_cap); mode "deposit" returns
    (dose[nX,nY,nZ] float64, active_at_cap).
    """
    xv, yv, zv = (np.asarray(grid[k], dtype=np.float64) for k in ("xv", "yv", "zv"))
    nx, ny, nz = xv.size, yv.size, zv.size
    twod = nz == 1
    vmax = np.array([xv.max(), yv.max(), zv.max()])
    vmin = np.array([xv.min(), yv.min(), zv.min()])
    voxel = np.array([xv[1] - xv[0], yv[1] - yv[0], np.inf if twod else zv[1] - zv[0]])
    span = vmax - vmin
    with np.errstate(divide="ignore"):
        norm = 2.0 / span
    if not np.isfinite(norm[2]):
        norm[2] = 0.0
    cfg = _RayCfg()
    cfg.nx, cfg.ny, cfg.nz = nx, ny, nz
    for d in range(3):
        cfg.span[d], cfg.xmax[d], cfg.xmin[d] = span[d], vmax[d], vmin[d]
        cfg.voxel[d], cfg.norm[d] = voxel[d], norm[d]
    cfg.h32 = float(np.float32(step_size))
    cfg.h_idx = float(step_size / voxel[0])
    cfg.max_steps = int(max_num_step)
    cfg.check_every = int(check_every)
    cfg.twod = int(twod)
    keep = []
    cfg.n_kind = n_kind
    cfg.n_sur = n_sur
    if n_kind == 1:
        ng = _f64(n_grid)
        gg = _f64(grad_grid) if grad_grid is not None else central_difference(ng, voxel)
        gg = _f64(gg)
        keep += [ng, gg]
        cfg.n_grid, cfg.g_grid = _p(ng), _p(gg)
    cfg.a_kind, cfg.a_val, cfg.a_R = a_kind, a_val, a_R
    if a_kind == 3:
        ag = _f64(a_grid)
        keep.append(ag)
        cfg.a_grid = _p(ag)
    ab = _f64(absorb if absorb is not None else np.ones((nx, ny, nz)))
    keep.append(ab)
    cfg.absorb = _p(ab)
    x0 = np.ascontiguousarray(x0, np.float32)
    v0 = np.ascontiguousarray(v0, np.float32)
    nr = x0.shape[0]
    lib = _load()
    if mode == "integrate":
        ff = _f64(f).reshape(nx, ny, nz)
        out = np.empty(nr, np.float32)
        act = lib.orc_ray_trace(ctypes.byref(cfg), _p(x0, ctypes.c_float), _p(v0, ctypes.c_float),
                                float(energy0), nr, 0, _p(ff), None, _p(out, ctypes.c_float), None)
        return out, act
    gin = np.ascontiguousarray(g, np.float32).ravel()
    dose = np.empty((nx, ny, nz))
    act = lib.orc_ray_trace(ctypes.byref(cfg), _p(x0, ctypes.c_float), _p(v0, ctypes.c_float),
                            float(energy0), nr, 1, None, _p(gin, ctypes.c_float), None, _p(dose))
    return dose, act


def setup_rays_parallel(xv, yv, zv, angles_deg, inclination_deg=0.0, ray_density=1.0):
    """float32 numpy restatement of RayState.setupRaysParallel (pyTorchRayTrace.py:1515-1666)."""
    import torch

    real_nX, real_nY, real_nZ = xv.size, yv.size, zv.size
    ang = np.asarray(angles_deg) * np.pi / 180.0
    incl = (inclination_deg or 0.0) * np.pi / 180.0
    if real_nZ == 1:
        shape = (round(max(real_nX, real_nY) * ray_density), ang.size, real_nZ)
    else:
        shape = (round(max(real_nX, real_nY) * ray_density), ang.size, max(round(real_nZ * ray_density), 1))
    n0min = min(np.amin(xv), np.amin(yv))
    n0max = max(np.amax(xv), np.amax(yv))
    n0 = np.linspace(n0min, n0max, shape[0])
    n2 = np.linspace(np.amin(zv), np.amax(zv), shape[2])
    off = np.sqrt(n0max ** 2 + np.amax(zv) ** 2)
    t = lambda a: torch.as_tensor(a, dtype=torch.float32)
    inc = t(incl)
    G0, G1, G2 = torch.meshgrid(t(n0), t(ang), t(n2), indexing="ij")
    G0, G1, G2 = G0.ravel(), G1.ravel(), G2.ravel()
    x0 = torch.empty((G0.numel(), 3), dtype=torch.float32)
    x0[:, 0] = off * torch.cos(G1) * torch.cos(inc)
    x0[:, 1] = off * torch.sin(G1) * torch.cos(inc)
    x0[:, 2] = off * torch.sin(inc)
    x0[:, 0] += -G0 * torch.sin(G1) - G2 * torch.cos(G1) * torch.sin(inc)
    x0[:, 1] += G0 * torch.cos(G1) - G2 * torch.sin(G1) * torch.sin(inc)
    x0[:, 2] += G2 * torch.cos(inc)
    v0 = torch.empty((G0.numel(), 3), dtype=torch.float32)
    v0[:, 0] = -torch.cos(G1) * torch.cos(inc)
    v0[:, 1] = -torch.sin(G1) * torch.cos(inc)
    v0[:, 2] = -torch.sin(inc)
    return x0.numpy(), v0.numpy(), shape


# --------------------------------------------------------------------------
# optimizer helpers (numpy restatements, float64)
# --------------------------------------------------------------------------

def clip_to_circle(x):
    """vamtoolbox/util/data.py:14-40 (returns a copy)."""
    x = np.array(x, copy=True)
    cy, cx = np.meshgrid(np.linspace(-1, 1, x.shape[0]), np.linspace(-1, 1, x.shape[1]))
    m = cx ** 2 + cy ** 2 > 1
    if x.ndim == 2:
        x[m] = 0
    else:
        x[np.broadcast_to(m[..., None], x.shape)] = 0
    return x


def circle_mask(shape):
    """vamtoolbox/geometry.py:682-711 (2-D mask, broadcast over z)."""
    cy, cx = np.meshgrid(np.linspace(-1, 1, shape[0]), np.linspace(-1, 1, shape[1]))
    return cx ** 2 + cy ** 2 <= 1


def response_tables(A=0.0, K=1.0, B=25.0, M=0.5, nu=1.0, n_pts=512, lo=0.0, hi=1.0):
    """ResponseModel(type='interpolation', form='gen_log_fun') tables (response.py:105-118, 191-218)."""
    f = np.linspace(lo, hi, n_pts)
    e = np.exp(-B * (f - M))
    m = A + (K - A) / (1 + e) ** (1 / nu)
    dm = (1 / (K - A)) ** nu * (B / nu) * (m - A) ** (nu + 1) * e
    return f, m, dm


def bclp_dose_pass(dose, target, f_tab, m_tab, dm_tab, eps, weight, p):
    """BCLP.py:293-437 state update for one dose (float64 numpy)."""
    mapped = np.interp(dose, f_tab, m_tab, left=m_tab[0], right=m_tab[-1])
    e = mapped - target
    eb = np.abs(e) - eps
    v = eb > 0
    loss_sum = np.sum(v * weight * np.abs(eb) ** p)
    dm = np.interp(dose, f_tab, dm_tab, left=dm_tab[0], right=dm_tab[-1])
    operand = v * weight * (np.abs(eb) ** (p - 1)) * np.sign(e) * dm
    v0 = np.abs(e) > 0
    stats = np.array([
        loss_sum, np.sum(v), np.sum(v0), np.sum(v * np.abs(eb)), np.sum(np.abs(e)),
        np.sum(v * eb ** 2), np.sum(e ** 2), np.amax(v * np.abs(eb)), np.amax(v0 * np.abs(e)),
    ])
    return mapped, operand, stats


def calc_ver(x, gel, void):
    """metrics.py:47-76."""
    mn = np.min(x[gel])
    return np.sum(x[void] >= mn) / (np.sum(gel) + np.sum(void))
