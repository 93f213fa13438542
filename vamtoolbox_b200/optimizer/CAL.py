"""Computed axial lithography (CAL) gradient descent: the reference's vamtoolbox/optimizer/CAL.py.

Loop (CAL.py:147-195): x_thresh = sigmoid(x - d_h, g); delta_b = A.forward(x_thresh - target);
b = clip(b - lr (delta_b (1-m) + delta_b_prev m / (1 - m^(it+1))), 0); x = A.backward(b) / max;
VER per iteration.  engine="device" keeps x unnormalised with max(x) as a
device scalar read by the threshold kernel, records VER into a device log and,
without momentum or an exit threshold, replays one CUDA graph per iteration
(bit-depth quantisation runs the host loop).
"""
from __future__ import annotations

import time

import numpy as np
import torch

from .. import geometry, metrics
from ..fused import Workspace, capture, to_host_f64
from ..projectorconstructor import projectorconstructor
from ..util import data as udata


def _threshold_reconstruction(x, target_geo, sigmoid):
    """CAL.py:39-114 (used when d_h is None)."""
    lo, hi = np.amin(x), np.amax(x)
    tests = np.linspace(lo, hi, 100)
    gel, void = target_geo.gel_inds, target_geo.void_inds
    score = np.zeros(tests.size)
    for i, t in enumerate(tests):
        th = np.where(x > t, 1, 0)
        score[i] = np.sum(th[gel]) / np.sum(gel) - np.sum(th[void]) / np.sum(void)
    thr = tests[np.argmax(score)]
    return 1 / (1 + np.exp(-(float(sigmoid) * (x - thr)))), thr


def _cal_host(target_geo, proj_geo, options, A=None):
    A = A if A is not None else projectorconstructor(target_geo, proj_geo)
    err = np.full(options.n_iter, np.nan)
    iter_times = np.zeros(options.n_iter)
    t0 = time.perf_counter()
    b = A.forward(target_geo.array)
    b = np.clip(udata.filterSinogram(b, options.filter), a_min=0, a_max=None)
    db_prev = np.zeros_like(b)
    x = A.backward(b)
    x = x / np.max(x)
    err[0] = metrics.calcVER(target_geo, x)
    iter_times[0] = time.perf_counter() - t0
    x_opt, b_opt = x, b
    for it in range(1, options.n_iter):
        if options.d_h is not None:
            xt = udata.sigmoid(x - options.d_h, options.sigmoid)
        else:
            xt, _ = _threshold_reconstruction(x, target_geo, options.sigmoid)
        db = A.forward(xt - target_geo.array)
        m = options.momentum
        grad = db * (1 - m) + db_prev * m / (1 - m ** (it + 1))
        b = np.clip(b - options.learning_rate * grad, a_min=0, a_max=None)
        if options.bit_depth is not None:
            b = udata.discretize(b, options.bit_depth, [0.0, np.max(b)])
        x = A.backward(b)
        x = x / np.amax(x)
        db_prev = db
        x_opt, b_opt = x, b
        err[it] = metrics.calcVER(target_geo, x)
        iter_times[it] = time.perf_counter() - t0
        if options.exit_param is not None and err[it] <= options.exit_param:
            break
    b_opt = np.where(b_opt < 0, 0, b_opt)
    b_opt = b_opt / np.amax(b_opt)
    x_opt = A.backward(b_opt)
    x_opt = x_opt / np.amax(x_opt)
    return (geometry.Sinogram(b_opt, proj_geo, options), geometry.Reconstruction(x_opt, proj_geo, options), err)


class CALDevice:
    """Device state and fused kernels of the CAL loop (CAL.py:147-195).

    The reconstruction x is kept unnormalised with max(x) as a device
    scalar.  ``step(it)`` issues one iteration on the current stream: the
    sigmoid threshold of x / max(x) against the target, the forward
    projection of the residual, the (momentum) sinogram update clipped at
    zero, the backprojection, its maximum, VER and the log append.  Nothing
    is allocated and nothing syncs, so a step is captured once as a CUDA
    graph when the momentum is zero.
    """

    def __init__(self, target_geo, proj_geo, options, A, ops=None):
        from ._device_ops import device_ops

        self.options = options
        # the projector's device entry points: back(b, out), fwd(x, out) (parallel beam, vector geometry)
        self.back, self.fwd, vs, ss, dev = ops if ops is not None else device_ops(A, target_geo, options.n_iter)
        self.device = dev
        ws = self.ws = Workspace(dev)
        self.tgt = torch.as_tensor(np.ascontiguousarray(np.atleast_3d(target_geo.array), dtype=np.float32),
                                   device=dev)
        self.mask = torch.as_tensor(metrics.region_mask(target_geo).reshape(vs), device=dev)
        n_iter = options.n_iter
        self.err_log = torch.full((max(n_iter, 1),), float("nan"), dtype=torch.float32, device=dev)
        self.counter = torch.zeros(1, dtype=torch.int32, device=dev)
        self.ver, self.xmax = ws.scalar(), ws.scalar()
        # initial sinogram: forward, filter (cuFFT), clip
        b = torch.empty(ss, dtype=torch.float32, device=dev)
        self.fwd(self.tgt, b)
        self.b = udata.filterSinogram_t(b, options.filter, lo=0.0)
        self.x = torch.empty(vs, dtype=torch.float32, device=dev)
        self.back(self.b, self.x)
        ws.max(self.x, self.xmax)
        ws.ver(self.x, self.mask, self.ver)
        ws.append(self.ver, self.err_log, self.counter)
        self.xt = torch.empty(vs, dtype=torch.float32, device=dev)
        self.db = torch.empty(ss, dtype=torch.float32, device=dev)
        self.db_prev = torch.zeros(ss, dtype=torch.float32, device=dev)
        self.m, self.lr = float(options.momentum), float(options.learning_rate)

    def step(self, it):
        o, ws = self.options, self.ws
        ws.cal_threshold(self.x, self.xmax, self.tgt, o.d_h, o.sigmoid, self.xt)
        self.fwd(self.xt, self.db)
        ws.cal_update(self.b, self.db, self.db_prev if self.m != 0 else None, self.lr, self.m, it)
        self.back(self.b, self.x)
        ws.max(self.x, self.xmax)
        ws.ver(self.x, self.mask, self.ver)
        ws.append(self.ver, self.err_log, self.counter)


def minimizeCAL(target_geo, proj_geo, options):
    from ._device_ops import device_ops

    A = projectorconstructor(target_geo, proj_geo)
    ops = None
    if getattr(options, "engine", "device") != "host" and options.d_h is not None and options.bit_depth is None:
        ops = device_ops(A, target_geo, options.n_iter)
    # the set-up filters the sinogram along its detector axis: projectors with a (detector, angle, z)
    # sinogram (parallel beam, vector geometry); the ray tracer's and algebraic propagator's flat ones
    # take the host loop
    if ops is None or len(ops[3]) != 3:
        return _cal_host(target_geo, proj_geo, options, A)
    c = CALDevice(target_geo, proj_geo, options, A, ops)
    dev, ws, n_iter, m = c.device, c.ws, options.n_iter, c.m
    st = torch.cuda.current_stream(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    done = 0
    graphable = m == 0 and options.bit_depth is None and options.exit_param is None
    if graphable and n_iter > 2:
        gr = capture(lambda: c.step(1), dev)
        ev0.record(st)
        for _ in range(1, n_iter):
            gr.replay()
        ev1.record(st)
        done = n_iter - 1
    else:
        ev0.record(st)
        for it in range(1, n_iter):
            c.step(it)
            done += 1
            if m != 0:
                c.db_prev.copy_(c.db)
            if options.exit_param is not None and float(c.ver.item()) <= options.exit_param:
                break
        ev1.record(st)
    # final positivity / normalisation / reconstruction (CAL.py:197-208)
    b, xmax = c.b, c.xmax
    bmax = ws.scalar()
    b.clamp_(min=0)
    ws.max(b, bmax)
    ws.scale(b, bmax)
    x_opt = torch.empty_like(c.x)
    c.back(b, x_opt)
    ws.max(x_opt, xmax)
    ws.scale(x_opt, xmax)
    err = c.err_log.double().cpu().numpy()
    err = np.where(np.arange(err.size) < int(c.counter.item()), err, np.nan)
    # device time per iteration of the loop (CUDA events on the engine's stream)
    options.device_iteration_ms = ev0.elapsed_time(ev1) / done if done else None
    b_h, x_h = to_host_f64(b, x_opt)
    return geometry.Sinogram(b_h, proj_geo, options), geometry.Reconstruction(x_h, proj_geo, options), err
