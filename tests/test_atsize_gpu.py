"""Parity at the benchmark sizes: the device iterations at the exact sizes the
bench times, checked against the float64 oracle on z-slab samples.

z-slices are independent for the vertical parallel beam, so the oracle runs
the projectors on a slab of 16 slices (seconds) while the device runs the
whole volume, i.e. the same kernel instances and launch shapes as the timed
configuration.  Elementwise passes and reductions are checked on the whole
volume from the device's own inputs.  Tolerances: relL2 <= 1e-5 for
projector products, <= 1e-4 for optimizer state and ray-traced quantities
(float32 atomics order), as the target requires.
"""
import numpy as np
import pytest
import torch

import bench
from oracle import iterations as OI
from oracle import oracle as O
from tests.conftest import relL2

pytestmark = pytest.mark.gpu

TOL_PROJ = 1e-5
TOL_STATE = 1e-4
SLAB = 16


def h(t):
    return t.double().cpu().numpy()


def _slab(n):
    z0 = n // 2 - SLAB // 2
    return slice(z0, z0 + SLAB)


def _bclp_case(tg, pg, opts):
    from vamtoolbox_b200.optimizer.BCLP import BCLPNorm

    it = BCLPNorm(tg, pg, opts).device_iteration()
    g = h(it.g)
    it.step()
    torch.cuda.synchronize()
    d = {"g": g, "dose": h(it.dose), "mapped": h(it.mapped), "operand": h(it.operand), "fwd": h(it.grad),
         "stats": h(it.stats), "g_new": h(it.g)}
    ang = np.asarray(pg.angles, np.float64)
    mask = np.asarray(pg.absorption_mask)[:, :, 0] if pg.absorption_mask is not None else None
    absn = None if mask is None else ("mask", mask)
    zs = _slab(tg.array.shape[2])
    # backprojection (R2) on a slab, from the same g
    dose_o = O.parallel_backward_ref(d["g"][:, :, zs], ang, absorption=absn)
    assert relL2(d["dose"][:, :, zs], dose_o) < TOL_PROJ
    # fused dose pass on the whole volume, from the device's dose
    rm = opts.response_model
    mapped_o, operand_o, stats_o = O.bclp_dose_pass(d["dose"], np.asarray(tg.array, np.float64), rm.interp_f_0,
                                                    rm.interp_map_0, rm.interp_dmapdf_0, opts.eps, opts.weight, opts.p)
    assert relL2(d["mapped"], mapped_o) < TOL_STATE
    assert relL2(d["operand"], operand_o) < TOL_STATE
    for k in (0, 1, 2, 3, 4, 5, 6, 7, 8):
        assert abs(d["stats"][k] - stats_o[k]) <= TOL_STATE * max(abs(stats_o[k]), 1e-30), (k, d["stats"][k], stats_o[k])
    # forward (R1) of the device's operand on a slab
    fwd_o = O.parallel_forward(d["operand"][:, :, zs], ang, absorption=absn)
    assert relL2(d["fwd"][:, :, zs], fwd_o) < TOL_PROJ
    # clamped update on the whole sinogram, from the device's forward and loss sum
    g_o = OI.bclp_update(d["g"], d["fwd"], d["stats"], opts.p, opts.q, opts.learning_rate, opts.blb, opts.bub)
    assert relL2(d["g_new"], g_o) < TOL_STATE
    # elementwise: within one float32 rounding of g_new plus 1e-5 of the step itself (the step lr * grad is
    # far below g, so its relative error is bounded by g's float32 rounding, not by the kernel)
    err = np.abs(d["g_new"] - g_o)
    assert np.all(err <= 2.0 ** -23 * np.abs(g_o) + 1e-5 * np.abs(g_o - d["g"]) + 1e-30)


def test_bclp_iteration_at_256cube_360_absorbing():
    tg, pg = bench.build_problem(256, 360, seed=1000)
    _bclp_case(tg, pg, bench.bclp_options(4))


@pytest.mark.parametrize("p", [2, 4])
def test_grayscale_bclp_iteration_at_192cube_720(p):
    _bclp_case(*bench.config_gray_bclp(4, p=p))


def test_osmo_half_step_at_256cube_360_absorbing():
    from vamtoolbox_b200.optimizer.OSMO import OSMODevice
    from vamtoolbox_b200.projectorconstructor import projectorconstructor

    tg, pg, opts = bench.config_osmo(4)
    it = OSMODevice(tg, pg, opts, projectorconstructor(tg, pg))
    x0, xm0 = h(it.x), h(it.xm)
    it.half(False)
    torch.cuda.synchronize()
    xm, b, x = h(it.xm), h(it.b), h(it.x)
    bmax, xmax = float(it.bmax.item()), float(it.xmax.item())
    # model update (void voxels lowered by max(x - d_l, 0)) on the whole volume
    xm_o = xm0.copy()
    dd = np.maximum(x0[tg.void_inds] - opts.d_l, 0)
    xm_o[tg.void_inds] -= dd
    assert relL2(xm, xm_o) < TOL_STATE
    ang = np.asarray(pg.angles, np.float64)
    absn = ("mask", np.asarray(pg.absorption_mask)[:, :, 0])
    zs = _slab(256)
    # forward of the model on a slab, against the device's sinogram before its normalisation
    b_raw = O.parallel_forward(xm[:, :, zs], ang, absorption=absn)
    assert relL2(b[:, :, zs] * bmax, np.maximum(b_raw, opts.inhibition * bmax)) < TOL_PROJ
    assert bmax >= b_raw.max() * (1 - 1e-6)
    # backprojection of the normalised sinogram on a slab, against the device's before its normalisation
    x_raw = O.parallel_backward_ref(b[:, :, zs], ang, absorption=absn)
    assert relL2(x[:, :, zs] * xmax, np.maximum(x_raw, 0)) < TOL_PROJ
    assert xmax >= x_raw.max() * (1 - 1e-6)


def test_cal_iteration_at_363sq_360():
    from vamtoolbox_b200.optimizer.CAL import CALDevice
    from vamtoolbox_b200.projectorconstructor import projectorconstructor

    tg, pg, opts = bench.config_cal_2d(4)
    c = CALDevice(tg, pg, opts, projectorconstructor(tg, pg))
    x0, b0 = h(c.x), h(c.b)
    c.step(1)
    torch.cuda.synchronize()
    xr, br, ver = OI.cal_step(x0, b0, np.atleast_3d(tg.array), np.atleast_3d(tg.gel_inds), np.atleast_3d(tg.void_inds),
                              np.asarray(pg.angles, np.float64), opts.d_h, opts.sigmoid, opts.learning_rate)
    xd = h(c.x)
    assert relL2(h(c.b), br) < TOL_STATE
    assert relL2(xd / xd.max(), xr) < TOL_STATE
    n = np.sum(tg.gel_inds) + np.sum(tg.void_inds)
    assert abs(float(c.ver.item()) - ver) * n <= 1.0 + 1e-9


def test_ray_tracer_block_of_angles_at_128cube_360():
    tg, pg, cv, nx, ax = bench.ray_problem(128, 360)
    from vamtoolbox_b200.projector.pyTorchRayTrace import PyTorchRayTracingPropagator

    P = PyTorchRayTracingPropagator(tg, pg)
    assert P.plan.max_num_step == 384
    r = bench.ray_chunk_parity(P.plan, cv, nx, ax, np.asarray(pg.angles), first=88, count=8)
    assert r["relL2"]["integrate"] < TOL_STATE, r
    assert r["relL2"]["deposit"] < TOL_STATE, r
