"""Seeded synthetic targets with the shapes of the benchmark workloads.

The reference ships no datasets; these generators produce the target classes
the benchmark configurations describe (binary unions of ellipses /
ellipsoids / cylinders inside a vial, smoothed-noise grayscale targets,
graded-index media) from a numpy Generator seed.
"""
from __future__ import annotations

import numpy as np


def ellipses_2d(n=256, seed=0, radius=120.0):
    """Union of 3-8 ellipses minus 2-4 circular holes inside a disk; semi-axes 10-80 px and holes
    4-20 px at the default radius of 120 px, scaled with the radius otherwise."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[:n, :n] - (n - 1) / 2
    img = np.zeros((n, n), dtype=bool)
    k = radius / 120.0
    for _ in range(rng.integers(3, 9)):
        a, b = rng.uniform(10, 80, 2) * k
        r = rng.uniform(0, max(radius - max(a, b) * 0.5, 0.0))
        phi = rng.uniform(0, 2 * np.pi)
        cx, cy = r * np.cos(phi), r * np.sin(phi)
        th = rng.uniform(0, np.pi)
        xr = (x - cx) * np.cos(th) + (y - cy) * np.sin(th)
        yr = -(x - cx) * np.sin(th) + (y - cy) * np.cos(th)
        img |= (xr / a) ** 2 + (yr / b) ** 2 <= 1
    for _ in range(rng.integers(2, 5)):
        rr = rng.uniform(4, 20) * k
        cx, cy = rng.uniform(-radius / 2, radius / 2, 2)
        img &= ~((x - cx) ** 2 + (y - cy) ** 2 <= rr ** 2)
    img &= x ** 2 + y ** 2 <= radius ** 2
    return img.astype(np.float64)


def ellipsoids_3d(n=256, nz=None, seed=0, radius=120.0):
    """Union of 5-12 random ellipsoids and z-cylinders inside a radius-`radius` vial."""
    nz = n if nz is None else nz
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[:n, :n] - (n - 1) / 2
    z = np.arange(nz) - (nz - 1) / 2
    vol = np.zeros((n, n, nz), dtype=bool)
    for _ in range(rng.integers(5, 13)):
        cyl = rng.uniform() < 0.4
        a, b = rng.uniform(0.05, 0.35, 2) * n
        c = rng.uniform(0.1, 0.4) * nz
        r = rng.uniform(0, radius - max(a, b) * 0.5)
        phi = rng.uniform(0, 2 * np.pi)
        cx, cy = r * np.cos(phi), r * np.sin(phi)
        cz = rng.uniform(-0.3, 0.3) * nz
        th = rng.uniform(0, np.pi)
        xr = (x - cx) * np.cos(th) + (y - cy) * np.sin(th)
        yr = -(x - cx) * np.sin(th) + (y - cy) * np.cos(th)
        q = (xr / a) ** 2 + (yr / b) ** 2
        for k, zz in enumerate(z):
            if cyl:
                if abs(zz - cz) <= c:
                    vol[:, :, k] |= q <= 1
            else:
                t = 1 - ((zz - cz) / c) ** 2
                if t > 0:
                    vol[:, :, k] |= q <= t
    vol &= (x ** 2 + y ** 2 <= radius ** 2)[:, :, None]
    return vol.astype(np.float64)


def _smooth(a, sigma):
    from scipy.ndimage import gaussian_filter

    return gaussian_filter(a, sigma)


def grayscale_3d(n=192, seed=0, sigma=4.0):
    """Gaussian-smoothed noise quantised to {0, 0.5, 1} plus a smooth ramp region."""
    rng = np.random.default_rng(seed)
    f = _smooth(rng.standard_normal((n, n, n)), sigma)
    f = (f - f.mean()) / (f.std() + 1e-12)
    t = np.where(f > 0.6, 1.0, np.where(f > -0.2, 0.5, 0.0))
    y, x = np.mgrid[:n, :n] - (n - 1) / 2
    ramp = np.clip((x + n / 4) / (n / 2), 0, 1)
    region = ((x / (0.3 * n)) ** 2 + (y / (0.15 * n)) ** 2 <= 1)
    for k in range(n // 3, 2 * n // 3):
        t[:, :, k] = np.where(region, ramp, t[:, :, k])
    r2 = x ** 2 + y ** 2
    t[r2 > ((n - 1) / 2) ** 2] = 0
    return t


def graded_index(coord_vec, seed=0, n0=1.50, dn=0.02, pert=0.005, sigma=6.0):
    """n = n0 + dn (r/R)^2 + smooth perturbation of amplitude +-pert."""
    rng = np.random.default_rng(seed)
    xg, yg, _ = np.meshgrid(*coord_vec, indexing="ij")
    R = np.amax(coord_vec[0])
    p = _smooth(rng.standard_normal(xg.shape), sigma)
    p = pert * p / (np.abs(p).max() + 1e-12)
    return n0 + dn * (xg ** 2 + yg ** 2) / R ** 2 + p


def smooth_attenuation(coord_vec, alpha0, seed=0, amp=0.3, sigma=6.0):
    """alpha = alpha0 (1 + amp * smooth noise in [-1, 1])."""
    rng = np.random.default_rng(seed + 1)
    shape = tuple(len(c) for c in coord_vec)
    p = _smooth(rng.standard_normal(shape), sigma)
    p = p / (np.abs(p).max() + 1e-12)
    return alpha0 * (1 + amp * p)
