"""CPU oracle of the output formats: projector frames and fan-beam rebinning.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by bench.py's CPU-baseline legs, as the checker or the timed CPU
baseline, never by the product package ``vamtoolbox_b200``.

numpy restatements, each pinned against the reference's own outputs in
tests/golden/formats.npz (tests/golden/make_golden.py runs the reference):

* ``image_frames`` follows ImageSeq.__init__ (vamtoolbox/imagesequence.py:
  85-174) with _invertU / _invertV (:358-365), _rotate (:396-401, scipy's
  ndimage.rotate order 1 restated in ``rotate_planes``), _scaleSize
  (:368-378, OpenCV's bilinear resize restated in ``resize_planes``),
  np.percentile, _scaleIntensity / _truncateIntensity (:381-393), the cast
  and _insertImage / _arrayInsertImage (:296-355).  The two third-party
  interpolations agree with the reference to a few ulps (their compiled
  kernels round in an order that is not published); everything else is the
  reference's arithmetic.
* ``rebin_fan`` follows rebinFanBeam (vamtoolbox/geometry.py:736-944) with
  scipy's interpn (method 'linear', fill 0) restated; bit-exact.
"""
from __future__ import annotations

import numpy as np
from scipy import special


def rotate_planes(sino, angle_deg):
    """ndimage.rotate(sino, angle, axes=(0, 2), reshape=True, order=1, mode='constant').

    Output (o0, o1) samples the input plane at c = rot @ o + offset, computed
    as (m00*o0 + off0) + m01*o1; zero when c0 is outside [0, nR-1] or c1 outside
    [0, nZ-1]; order-1 spline sum ((x * w0) * w1) over the corners in the
    order (lo,lo), (lo,hi), (hi,lo), (hi,hi).  Result in the input dtype.
    """
    sino = np.asarray(sino)
    n_r, n_a, n_z = sino.shape
    c, s = special.cosdg(angle_deg), special.sindg(angle_deg)
    rot = np.array([[c, s], [-s, c]])
    iy, ix = n_r, n_z
    bounds = rot @ [[0, 0, iy, iy], [0, ix, 0, ix]]
    o_r, o_z = (np.ptp(bounds, axis=1) + 0.5).astype(int)
    off = (np.array([n_r, n_z]) - 1) / 2 - rot @ ((np.array([o_r, o_z]) - 1) / 2)
    o0, o1 = np.meshgrid(np.arange(o_r, dtype=float), np.arange(o_z, dtype=float), indexing="ij")
    c0 = (rot[0, 0] * o0 + off[0]) + rot[0, 1] * o1
    c1 = (rot[1, 0] * o0 + off[1]) + rot[1, 1] * o1
    inside = (c0 >= 0) & (c0 <= n_r - 1) & (c1 >= 0) & (c1 <= n_z - 1)
    f0, f1 = np.floor(c0), np.floor(c1)
    t0, t1 = c0 - f0, c1 - f1
    a0, a1 = 1 - t0, 1 - t1
    i0 = np.clip(f0.astype(np.int64), 0, n_r - 1)
    i1 = np.clip(f1.astype(np.int64), 0, n_z - 1)
    j0 = np.minimum(i0 + 1, n_r - 1)
    j1 = np.minimum(i1 + 1, n_z - 1)
    x = sino.astype(np.float64)
    out = np.zeros((o_r, n_a, o_z), dtype=sino.dtype)
    for a in range(n_a):
        p = x[:, a, :]
        v = (p[i0, i1] * a0) * a1
        v = v + (p[i0, j1] * a0) * t1
        v = v + (p[j0, i1] * t0) * a1
        v = v + (p[j0, j1] * t0) * t1
        out[:, a, :] = np.where(inside, v, 0.0)
    return out


def _axis_taps(n_src, n_dst):
    scale = 1.0 / (n_dst / n_src)
    fx = (np.arange(n_dst, dtype=np.float64) + 0.5) * scale - 0.5
    s = np.floor(fx)
    fx = fx - s
    s = s.astype(np.int64)
    lo = s < 0
    fx[lo], s[lo] = 0.0, 0
    hi = s >= n_src - 1
    fx[hi], s[hi] = 0.0, n_src - 1
    return s, np.minimum(s + 1, n_src - 1), fx


def resize_planes(sino, scale_factor):
    """_scaleSize: cv2.resize(plane, (new_w, new_h), INTER_LINEAR) per angle,
    collected in a float64 array (vamtoolbox/imagesequence.py:368-378).

    Half-pixel centres, edge clamp, z (plane width) interpolated first; float32
    planes use float32 weights and arithmetic, float64 planes float64.
    """
    sino = np.asarray(sino)
    n_r, n_a, n_z = sino.shape
    new_h, new_w = int(n_r * scale_factor), int(n_z * scale_factor)
    sz0, sz1, fz = _axis_taps(n_z, new_w)
    sr0, sr1, fr = _axis_taps(n_r, new_h)
    dt = np.float32 if sino.dtype == np.float32 else np.float64
    wz1, wr1 = fz.astype(dt), fr.astype(dt)
    wz0, wr0 = dt(1) - wz1, dt(1) - wr1
    out = np.zeros((new_h, n_a, new_w))
    for a in range(n_a):
        p = sino[:, a, :].astype(dt)
        r0 = p[sr0][:, sz0] * wz0 + p[sr0][:, sz1] * wz1
        r1 = p[sr1][:, sz0] * wz0 + p[sr1][:, sz1] * wz1
        out[:, a, :] = r0 * wr0[:, None] + r1 * wr1[:, None]
    return out


def _insert_bounds(cfg, s_u, s_v, v_off):
    u1 = int(cfg["N_u"] / 2 - cfg["u_offset"] - s_u / 2)
    u2 = int(cfg["N_u"] / 2 - cfg["u_offset"] + s_u / 2)
    v1 = int(cfg["N_v"] / 2 - cfg["v_offset"] - v_off - s_v / 2)
    v2 = int(cfg["N_v"] / 2 - cfg["v_offset"] - v_off + s_v / 2)
    if u1 < 0 or u2 > cfg["N_u"] or v1 < 0 or v2 > cfg["N_v"]:
        raise Exception("Image could not be inserted")
    return u1, u2, v1, v2


def config(N_u, N_v, **kw):
    """The ImageConfig fields as a dict, with the reference's defaults (:55-82)."""
    cfg = dict(N_u=N_u, N_v=N_v, rotate_angle=0.0, u_offset=0, v_offset=0, invert_u=False, invert_v=False,
               array_num=1, array_offset=0, normalization_percentile=None, intensity_scale=1.0, bit_depth=8,
               size_scale=1.0)
    cfg.update(kw)
    return cfg


def image_frames(sino, cfg, return_float=False):
    """Frames [nA][N_v][N_u] uint8 of ImageSeq(ImageConfig(**cfg), sino).images.

    With return_float=True also returns the sinogram after the plane
    transforms and the intensity chain, before the integer cast.
    """
    mod = np.copy(np.asarray(sino))
    if cfg["invert_u"]:
        mod = np.flip(mod, axis=0)
    if cfg["invert_v"]:
        mod = np.flip(mod, axis=2)
    if cfg["rotate_angle"] != 0.0:
        mod = rotate_planes(mod, cfg["rotate_angle"])
    if cfg["size_scale"] != 1.0:
        mod = resize_planes(mod, cfg["size_scale"])
    mx = 2 ** cfg["bit_depth"] - 1
    if cfg["normalization_percentile"] is not None:
        mod = mod / np.percentile(mod, cfg["normalization_percentile"]) * mx
    if cfg["intensity_scale"] != 1.0:
        mod = mod * cfg["intensity_scale"]
    bd = cfg["bit_depth"]
    dtype = np.uint8 if bd <= 8 else (np.uint16 if bd <= 16 else np.uint32)
    mod = np.minimum(mod, mx)
    with np.errstate(invalid="ignore"):
        q = mod.astype(dtype)
    n_r, n_a, n_z = q.shape
    frames = np.zeros((n_a, cfg["N_v"], cfg["N_u"]), dtype=np.uint8)
    if cfg["array_num"] == 1:
        offsets = [0]
    else:
        offsets = []
        for k in range(cfg["array_num"]):
            if cfg["array_num"] % 2 == 0:
                d = int(np.ceil((k + 1) / 2) * (-1) ** k)
                offsets.append(int(cfg["array_offset"] * d / 2 + cfg["v_offset"]))
            else:
                d = int(0 + np.ceil(k / 2) * (-1) ** (k + 1))
                offsets.append(int(cfg["array_offset"] * d + cfg["v_offset"]))
    for v_off in offsets:
        u1, u2, v1, v2 = _insert_bounds(cfg, n_r, n_z, v_off)
        # frame[a, v1:v2, u1:u2] = q[:, a, :].T, stored into uint8 (low byte)
        frames[:, v1:v2, u1:u2] = np.transpose(q, (1, 2, 0))
    if return_float:
        return frames, mod
    return frames


def rebin_fan(sino, angles, vial_width, N_screen, n_write, throw_ratio):
    """rebinFanBeam (vamtoolbox/geometry.py:736-944) with interpn restated.

    Returns the rebinned [vial_width][nA][nZ] array in the input dtype (the
    reference also pads its input in place; this function leaves it alone).
    """
    sino = np.asarray(sino)
    angles = np.asarray(angles)
    n_r, n_a, n_z = sino.shape
    vial_width = int(vial_width)
    trp = throw_ratio * N_screen[0]
    Rv = (vial_width / 2) * np.sqrt(1 + ((vial_width) / (2 * trp)) ** 2)
    xp = np.linspace(-vial_width / 2, vial_width / 2, vial_width)
    phi = np.arctan(xp / trp)
    xps = (xp - xp * np.sqrt(1 - (1 + (xp / trp) ** 2) * (1 - (Rv / trp) ** 2))) / (1 + (xp / trp) ** 2)
    theta10 = np.arcsin(xps / Rv)
    thetai = np.arcsin(xps / Rv) + phi
    thetat = np.arcsin((1 / n_write) * np.sin(thetai))
    thetav = theta10 - thetat
    thetavD = (180 / np.pi) * thetav
    Ts = 1 - ((1 * np.cos(thetai) - n_write * np.cos(thetat)) / ((1 * np.cos(thetai) + n_write * np.cos(thetat)))) ** 2
    Tp = 1 - ((1 * np.cos(thetat) - n_write * np.cos(thetai)) / ((1 * np.cos(thetat) + n_write * np.cos(thetai)))) ** 2
    T = (Ts + Tp) / 2
    T[T < 0] = 0
    xv = (xps * np.cos(thetav)) - (np.sin(thetav) * np.sqrt((Rv ** 2) - (xps ** 2)))
    d = np.gradient(xv)
    d[T < 0] = 0
    d[d < 0] = 0
    th = angles[None, :] + thetavD[:, None]
    mn, mxa = angles[0], angles[-1]
    dt = abs(angles[1] - angles[0])
    th[th > mxa] = th[th > mxa] - 360
    th[th < mn] = 360 + th[th < mn]
    th[th > mxa - dt] = mn
    pd = int((vial_width - n_r) / 2)
    b = sino
    if pd > 0:
        b = np.pad(b, ((pd, pd), (0, 0), (0, 0)))
    if b.shape[0] < vial_width:
        b = np.pad(b, ((0, 1), (0, 0), (0, 0)))

    def search(grid, x):
        i = np.clip(np.searchsorted(grid, x, side="left") - 1, 0, grid.size - 2)
        return i, (x - grid[i]) / (grid[i + 1] - grid[i]), (x < grid[0]) | (x > grid[-1])

    xs = np.broadcast_to(xv[:, None], th.shape)
    i0, y0, o0 = search(xp, xs)
    i1, y1, o1 = search(angles, th)
    oob = o0 | o1
    out = np.zeros_like(b)
    with np.errstate(divide="ignore", invalid="ignore"):
        tinv = 1 / T
        for z in range(n_z):
            v = b[..., z]
            r = (v[i0, i1] * (1 - y0) * (1 - y1) + v[i0, i1 + 1] * (1 - y0) * y1 + v[i0 + 1, i1] * y0 * (1 - y1)
                 + v[i0 + 1, i1 + 1] * y0 * y1)
            r = np.where(oob, 0.0, r)
            r = r * d[:, None]
            out[..., z] = tinv[:, None] * r
    return out


def select_pair(x, k0, k1):
    """The k0-th and k1-th smallest of x (NaN sorts last; any NaN gives NaN, NaN)."""
    x = np.asarray(x).ravel()
    if np.isnan(x).any():
        return np.array([np.nan, np.nan], dtype=x.dtype)
    s = np.sort(x)
    return np.array([s[k0], s[k1]], dtype=x.dtype)
