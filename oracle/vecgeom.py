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
