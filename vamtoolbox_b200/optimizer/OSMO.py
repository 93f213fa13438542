"""Object-space model optimisation (OSMO): the reference's vamtoolbox/optimizer/OSMO.py.

Per iteration (OSMO.py:36-109, 141-147): the model is lowered on void voxels
by max(x - d_l, 0) and raised on gel voxels by max(d_h - x, 0); after each
update b = A.forward(model) / max, floored at the inhibition level, and
x = max(A.backward(b) / max, 0).  engine="device" runs the two half steps as
fused kernels with device-side maxima and replays them as one CUDA graph.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from .. import geometry, metrics
from ..fused import Workspace, capture, to_device_f64, to_host_f64
from ..projectorconstructor import projectorconstructor
from ..util import data as udata


def _osmo_host(target_geo, proj_geo, options, A):
    err = np.full(options.n_iter, np.nan)
    inh = options.inhibition
    t0 = time.perf_counter()
    xm = np.real(udata.filterTargetOSMO(target_geo.array, options.filter))
    b = np.clip(A.forward(xm), 0, None)
    x = A.backward(b)
    x = x / np.amax(x)
    err[0] = metrics.calcVER(target_geo, x)

    def half(x, xm, gel):
        if gel:
            d = options.d_h - x[target_geo.gel_inds]
            d[d < 0] = 0
            xm[target_geo.gel_inds] = xm[target_geo.gel_inds] + d
        else:
            d = x[target_geo.void_inds] - options.d_l
            d[d < 0] = 0
            xm[target_geo.void_inds] = xm[target_geo.void_inds] - d
        b = A.forward(xm)
        b = b / np.amax(b)
        if options.bit_depth is not None:
            b = udata.discretize(b, options.bit_depth, [np.min(b), np.max(b)])
        b[b < inh] = inh
        xu = A.backward(b)
        xu = xu / np.amax(xu)
        xu[xu < 0] = 0
        return xu, b, xm

    for it in range(1, options.n_iter):
        x, _, xm = half(x, xm, False)
        x, b, xm = half(x, xm, True)
        err[it] = metrics.calcVER(target_geo, x)
        if options.exit_param is not None and err[it] <= options.exit_param:
            break
    b_opt = udata.discretize(b, options.bit_depth, [0.0, np.max(b)]) if options.bit_depth is not None else b
    return geometry.Sinogram(b_opt, proj_geo, options), geometry.Reconstruction(x, proj_geo, options), err


class OSMODevice:
    """Device state and fused kernels of the OSMO loop (OSMO.py:36-109, 141-147).

    ``half(gel)`` issues one half step on the current stream: the model
    update on void (gel False) or gel voxels, the forward projection, its
    device-side maximum and the normalisation floored at the inhibition
    level, the backprojection, its maximum and the normalisation floored at
    zero.  ``step()`` is one OSMO iteration (void half, gel half, VER, log
    append).  Nothing is allocated and nothing syncs, so ``capture()``
    records a step once as a CUDA graph.
    """

    def __init__(self, target_geo, proj_geo, options, A, ops=None):
        from ._device_ops import device_ops

        self.options = options
        self.A = A
        # the projector's device entry points: back(b, out), fwd(x, out) (parallel beam, vector geometry,
        # ray tracer, algebraic propagator)
        self.back, self.fwd, vs, ss, dev = ops if ops is not None else device_ops(A, target_geo, options.n_iter)
        self.device = dev
        ws = self.ws = Workspace(dev)
        self.mask = torch.as_tensor(metrics.region_mask(target_geo).reshape(vs), device=dev)
        n_iter = options.n_iter
        self.err_log = torch.full((max(n_iter, 1),), float("nan"), dtype=torch.float32, device=dev)
        self.counter = torch.zeros(1, dtype=torch.int32, device=dev)
        self.ver, self.xmax, self.bmax = ws.scalar(), ws.scalar(), ws.scalar()
        tgt = to_device_f64(target_geo.array, dev)
        self.xm = udata.filterTargetOSMO_t(tgt, options.filter).to(torch.float32).reshape(vs).contiguous()
        self.b = torch.empty(ss, dtype=torch.float32, device=dev)
        self.x = torch.empty(vs, dtype=torch.float32, device=dev)
        self.fwd(self.xm, self.b)
        self.b.clamp_(min=0)
        self.back(self.b, self.x)
        ws.max(self.x, self.xmax)
        ws.scale(self.x, self.xmax)
        ws.ver(self.x, self.mask, self.ver)
        ws.append(self.ver, self.err_log, self.counter)
        self.inh = float(options.inhibition)

    def half(self, gel):
        o, ws = self.options, self.ws
        ws.osmo_model(self.xm, self.x, None, self.mask, gel, o.d_h if gel else o.d_l)
        self.fwd(self.xm, self.b)
        ws.max(self.b, self.bmax)
        ws.scale(self.b, self.bmax, floor=self.inh)
        self.back(self.b, self.x)
        ws.max(self.x, self.xmax)
        ws.scale(self.x, self.xmax, floor=0.0)

    def step(self):
        self.half(False)
        self.half(True)
        self.ws.ver(self.x, self.mask, self.ver)
        self.ws.append(self.ver, self.err_log, self.counter)

    def capture(self):
        return capture(self.step, self.device)


def minimizeOSMO(target_geo, proj_geo, options):
    from ._device_ops import device_ops

    A = projectorconstructor(target_geo, proj_geo)
    ops = None
    if getattr(options, "engine", "device") != "host" and options.bit_depth is None:
        ops = device_ops(A, target_geo, options.n_iter)
    if ops is None:
        return _osmo_host(target_geo, proj_geo, options, A)
    it = OSMODevice(target_geo, proj_geo, options, A, ops)
    dev, n_iter = it.device, options.n_iter
    st = torch.cuda.current_stream(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    done = 0
    if options.exit_param is None and n_iter > 2:
        gr = it.capture()
        ev0.record(st)
        for _ in range(1, n_iter):
            gr.replay()
        ev1.record(st)
        done = n_iter - 1
    else:
        ev0.record(st)
        for _ in range(1, n_iter):
            it.step()
            done += 1
            if options.exit_param is not None and float(it.ver.item()) <= options.exit_param:
                break
        ev1.record(st)
    err = it.err_log.double().cpu().numpy()
    # device time per iteration of the loop (CUDA events on the engine's stream)
    options.device_iteration_ms = ev0.elapsed_time(ev1) / done if done else None
    err = np.where(np.arange(err.size) < int(it.counter.item()), err, np.nan)
    b_h, x_h = to_host_f64(it.b, it.x)
    return geometry.Sinogram(b_h, proj_geo, options), geometry.Reconstruction(x_h, proj_geo, options), err
