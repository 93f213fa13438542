"""Float64 oracle of whole optimizer iterations at the benchmark sizes.

TEST INFRASTRUCTURE ONLY: imported by tests/ and by bench.py's CPU-baseline
leg (which times these same calls), always as the checker, never by the
product package ``vamtoolbox_b200``.

Each function strings together the oracle's restated projectors
(oracle/vamoracle.c through oracle/oracle.py) and numpy restatements of the
reference's iteration bodies, in float64:

- ``bclp_iteration``: one BCLP gradient step, vamtoolbox/optimizer/BCLP.py:277-386
  (updateVariables / computeLoss / computeLossGradient) and :477-534
  (gradientDescent, imposeSinogramConstraints), with the projector pair the
  reference uses for the parallel beam (Projector3DParallel.py:113-207) and
  the absorption mask of geometry.py:161-193 applied to the forward's input
  and the backprojection's output.
- ``osmo_half``: one half step of OSMO, vamtoolbox/optimizer/OSMO.py:36-109.
- ``cal_step``: one CAL iteration without momentum, vamtoolbox/optimizer/CAL.py:147-195
  with util/data.py:9-11 (sigmoid) and metrics.py:47-76 (VER).
- ``ray_chunk``: integrate and deposit of one block of angles' rays,
  vamtoolbox/projector/pyTorchRayTrace.py:378-571 with the rays of
  RayState.setupRaysParallel (:1515-1666).

Since z-slices are independent for the vertical parallel beam, a z-slab of
the volume and of the sinogram is an exact sub-problem of every projector
call; only the global scalars (the BCLP loss, OSMO's maxima) couple slices.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


def _abs(mask):
    return None if mask is None else ("mask", np.asarray(mask, dtype=np.float64))


def bclp_iteration(g, target, angles, mask, tables, eps, weight, p, q, lr, blb=0.0, bub=None):
    """One BCLP iteration from sinogram g (float64).  tables = (f, map, dmap) of the response model's
    interpolation (response.py:105-118).  Returns dose, mapped, operand, fwd (the forward of the
    operand, before the loss prefactor), stats (the 9 loss / norm sums) and g_new."""
    g = np.asarray(g, dtype=np.float64)
    absn = _abs(mask)
    dose = O.parallel_backward_ref(g, angles, absorption=absn)
    mapped, operand, stats = O.bclp_dose_pass(dose, target, *tables, eps, weight, p)
    fwd = O.parallel_forward(operand, angles, absorption=absn)
    loss = stats[0] ** (q / p)
    grad = q * loss ** ((q - p) / q) * fwd if loss != 0 else fwd
    g_new = np.clip(g - lr * grad, blb, bub)
    return {"dose": dose, "mapped": mapped, "operand": operand, "fwd": fwd, "stats": stats, "g_new": g_new}


def bclp_update(g, fwd, stats, p, q, lr, blb=0.0, bub=None):
    """The clamped sinogram update of BCLP.py:477-534 from a given forward and loss sum."""
    loss = float(stats[0]) ** (q / p)
    grad = q * loss ** ((q - p) / q) * fwd if loss != 0 else fwd
    return np.clip(np.asarray(g, dtype=np.float64) - lr * grad, blb, bub)


def osmo_half(x, xm, gel, void, use_gel, d, angles, mask=None, inhibition=0.0):
    """One OSMO half step (OSMO.py:36-109): the model xm is lowered on void voxels by max(x - d_l, 0)
    (use_gel False) or raised on gel voxels by max(d_h - x, 0); b = forward(xm) / max, floored at the
    inhibition level; x = backward(b) / max, negatives zeroed.  Returns (x, b, xm), float64."""
    x = np.asarray(x, dtype=np.float64)
    xm = np.array(xm, dtype=np.float64, copy=True)
    absn = _abs(mask)
    if use_gel:
        dd = d - x[gel]
        dd[dd < 0] = 0
        xm[gel] = xm[gel] + dd
    else:
        dd = x[void] - d
        dd[dd < 0] = 0
        xm[void] = xm[void] - dd
    b = O.parallel_forward(xm, angles, absorption=absn)
    b = b / np.amax(b)
    b[b < inhibition] = inhibition
    xu = O.parallel_backward_ref(b, angles, absorption=absn)
    xu = xu / np.amax(xu)
    xu[xu < 0] = 0
    return xu, b, xm


def cal_step(x, b, target, gel, void, angles, d_h, sigmoid, lr):
    """One CAL iteration (CAL.py:147-195, momentum 0) from reconstruction x and sinogram b (float64):
    x_thresh = sigmoid(x / max(x) - d_h, g), delta_b = forward(x_thresh - target),
    b = max(b - lr delta_b, 0), x = backward(b) / max.  The reference keeps x normalised; dividing by the
    maximum first is the same.  Returns (x, b, VER)."""
    x = np.asarray(x, dtype=np.float64)
    xn = x / np.amax(x)
    xt = 1 / (1 + np.exp(-(xn - d_h) * (1 / sigmoid)))
    db = O.parallel_forward(xt - target, angles)
    b = np.clip(np.asarray(b, dtype=np.float64) - lr * db, 0, None)
    xu = O.parallel_backward_ref(b, angles)
    xu = xu / np.amax(xu)
    return xu, b, O.calc_ver(xu, gel, void)


def ray_chunk(cv, n_grid, a_grid, angles, first, count, f, g_rows, step_size, max_num_step):
    """Integrate f and deposit g over the rays of angles[first:first + count] (ray order (detector,
    angle, z) of pyTorchRayTrace.py:1629-1632; rows of these angles only).  The attenuation grid is
    both the path attenuation and the absorption at the grid points, the index grid's gradient is the
    central difference of medium.py:224-273.  Returns (integral [n0, count, nz] float32, dose float64,
    active rays at the step cap of the integrate pass)."""
    xv, yv, zv = cv
    x0, v0, shape = O.setup_rays_parallel(xv, yv, zv, np.asarray(angles)[first:first + count])
    kw = dict(step_size=step_size, max_num_step=max_num_step, n_kind=1, n_grid=n_grid, a_kind=3, a_grid=a_grid,
              absorb=a_grid)
    grid = dict(xv=xv, yv=yv, zv=zv)
    integral, act = O.ray_trace("integrate", grid, x0, v0, 1.0, f=f, **kw)
    dose, _ = O.ray_trace("deposit", grid, x0, v0, 1.0, g=np.asarray(g_rows, np.float32).ravel(), **kw)
    return integral.reshape(shape), dose, act
