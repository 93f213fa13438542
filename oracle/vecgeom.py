"""CPU oracle of the vector-geometry (ASTRA-model) parallel-beam projector.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()``
and bench.py's CPU legs, never by the product package ``vamtoolbox_b200``.

float64 numpy restatement of the model the reference's CUDA path hands to
ASTRA (vamtoolbox/projector/Projector3DParallelCUDA.py:13-72 with
genVectorsAstra.py:4-53), written from the geometry directly (pixel centre,
ray-plane intersection, 3x3 solve) rather than from the device's affine
tables.  Parity unpinned: ASTRA is absent here, so this oracle pins the
device kernels to the restated model, and the geometry vectors to the
reference's own genVectorsAstra (tests/golden/vecgeom.npz).
"""
from __future__ import annotations

import numpy as np


def _bilinear(plane, f0, f1):
    """Sample plane[n0][n1] at continuous indices (f0, f1), zero outside."""
    n0, n1 = plane.shape
    g0, g1 = np.floor(f0), np.floor(f1)
    t0, t1 = f0 - g0, f1 - g1
    i0, i1 = g0.astype(np.int64), g1.astype(np.int64)
    out = np.zeros(np.broadcast(f0, f1).shape)
    for d0, w0 in ((0, 1 - t0), (1, t0)):
        for d1, w1 in ((0, 1 - t1), (1, t1)):
            a, b = i0 + d0, i1 + d1
            ok = (a >= 0) & (a < n0) & (b >= 0) & (b < n1)
            val = np.where(ok, plane[np.clip(a, 0, n0 - 1), np.clip(b, 0, n1 - 1)], 0.0)
            out = out + w0 * w1 * val
    return out


def _centres(shape):
    return np.array([0.5 - n / 2.0 for n in shape])


def forward(vol, vectors, n_u, n_v):
    """Sinogram [n_u][nA][n_v] of vol [nY][nX][nZ] (Joseph-type, dominant-axis planes)."""
    vol = np.asarray(vol, dtype=np.float64)
    cen = _centres(vol.shape)
    vectors = np.asarray(vectors, dtype=np.float64).reshape(-1, 12)
    out = np.zeros((n_u, vectors.shape[0], n_v))
    cc, rr = np.meshgrid(np.arange(n_u), np.arange(n_v), indexing="ij")
    for a, q in enumerate(vectors):
        ray, d, u, v = q[0:3], q[3:6], q[6:9], q[9:12]
        P = (d[:, None, None] + (cc - n_u / 2 + 0.5)[None] * u[:, None, None]
             + (rr - n_v / 2 + 0.5)[None] * v[:, None, None])
        r = np.abs(ray)   # dominant axis: x on ties with y or z, then y on a tie with z
        ax = 0 if (r[0] >= r[1] and r[0] >= r[2]) else (1 if r[1] >= r[2] else 2)
        others = [b for b in range(3) if b != ax]
        acc = np.zeros((n_u, n_v))
        for s in range(vol.shape[ax]):
            t = (cen[ax] + s - P[ax]) / ray[ax]
            f = [P[b] + t * ray[b] - cen[b] for b in others]
            plane = np.take(vol, s, axis=ax)
            acc += _bilinear(plane, f[0], f[1])
        out[:, a, :] = acc * np.linalg.norm(ray) / abs(ray[ax])
    return out


def backward(sino, vectors, vol_shape):
    """Voxel-driven backprojection of sino [n_u][nA][n_v] onto vol_shape [nY][nX][nZ]."""
    sino = np.asarray(sino, dtype=np.float64)
    n_u, _, n_v = sino.shape
    cen = _centres(vol_shape)
    grids = np.meshgrid(*[np.arange(n) for n in vol_shape], indexing="ij")
    p = np.stack([g + c for g, c in zip(grids, cen)])          # voxel centres
    vectors = np.asarray(vectors, dtype=np.float64).reshape(-1, 12)
    out = np.zeros(vol_shape)
    for a, q in enumerate(vectors):
        ray, d, u, v = q[0:3], q[3:6], q[6:9], q[9:12]
        M = np.stack([u, v, ray], axis=1)
        sol = np.linalg.solve(M, (p - d[:, None, None, None]).reshape(3, -1)).reshape((3,) + tuple(vol_shape))
        fu = sol[0] + n_u / 2 - 0.5
        fv = sol[1] + n_v / 2 - 0.5
        out += _bilinear(sino[:, a, :], fu, fv)
    return out


# ---------------------------------------------------------------------------
# 2-D "line" model (vamtoolbox/projector/Projector2DParallelCUDA.py:7-45)
# ---------------------------------------------------------------------------

def _segment_in_square(p0, d, cx, cy):
    """Length of the line p0 + s d (|d| = 1) inside the unit square centred at (cx, cy)
    (Liang-Barsky clipping of an unbounded line)."""
    lo, hi = -np.inf * np.ones(np.broadcast(cx, cy).shape), np.inf * np.ones(np.broadcast(cx, cy).shape)
    for k, c in ((0, cx), (1, cy)):
        if abs(d[k]) < 1e-15:
            inside = np.abs(p0[k] - c) <= 0.5
            lo = np.where(inside, lo, np.inf)
            hi = np.where(inside, hi, -np.inf)
        else:
            s1 = (c - 0.5 - p0[k]) / d[k]
            s2 = (c + 0.5 - p0[k]) / d[k]
            lo = np.maximum(lo, np.minimum(s1, s2))
            hi = np.minimum(hi, np.maximum(s1, s2))
    return np.maximum(hi - lo, 0.0)


def line2d_matrix(n_y, n_x, angles_deg, n_t):
    """Dense system matrix [nT * nA][nY * nX] of the line model: row (d, a) holds the
    intersection lengths of ray (d, a) with every pixel, ASTRA's 2-D frame
    (pixel (i, j) at (j - nX/2 + 1/2, nY/2 - i - 1/2), bin d at d - nT/2 + 1/2 along
    (cos a, sin a), rays along (sin a, -cos a))."""
    ii, jj = np.meshgrid(np.arange(n_y), np.arange(n_x), indexing="ij")
    cx = (jj - n_x / 2 + 0.5).ravel()
    cy = (n_y / 2 - ii - 0.5).ravel()
    th = np.deg2rad(np.asarray(angles_deg, dtype=np.float64))
    M = np.zeros((n_t * th.size, n_y * n_x))
    for a, t in enumerate(th):
        u = np.array([np.cos(t), np.sin(t)])
        ray = np.array([np.sin(t), -np.cos(t)])
        for d in range(n_t):
            p0 = u * (d - n_t / 2 + 0.5)
            M[d * th.size + a] = _segment_in_square(p0, ray, cx, cy)
    return M


def _line2d_rows(n_y, n_x, angles_deg, n_t):
    """Yield (d, a, lengths over all pixels) for every ray, one row of line2d_matrix at a time."""
    ii, jj = np.meshgrid(np.arange(n_y), np.arange(n_x), indexing="ij")
    cx = (jj - n_x / 2 + 0.5).ravel()
    cy = (n_y / 2 - ii - 0.5).ravel()
    for a, t in enumerate(np.deg2rad(np.asarray(angles_deg, dtype=np.float64))):
        u = np.array([np.cos(t), np.sin(t)])
        ray = np.array([np.sin(t), -np.cos(t)])
        for d in range(n_t):
            yield d, a, _segment_in_square(u * (d - n_t / 2 + 0.5), ray, cx, cy)


def line2d_forward(img, angles_deg, n_t):
    """Sinogram [nT][nA] of img [nY][nX] under the line model (rows streamed, no dense matrix)."""
    img = np.asarray(img, dtype=np.float64)
    flat = img.ravel()
    out = np.zeros((n_t, np.size(angles_deg)))
    for d, a, row in _line2d_rows(img.shape[0], img.shape[1], angles_deg, n_t):
        out[d, a] = row @ flat
    return out


def line2d_backward(sino, angles_deg, shape):
    """Transpose of line2d_forward: sino [nT][nA] -> image of `shape`."""
    sino = np.asarray(sino, dtype=np.float64)
    out = np.zeros(shape[0] * shape[1])
    for d, a, row in _line2d_rows(shape[0], shape[1], angles_deg, sino.shape[0]):
        out += sino[d, a] * row
    return out.reshape(shape)
