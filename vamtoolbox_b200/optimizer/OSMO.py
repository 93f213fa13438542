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
from ..fused import Workspace, capture
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


def minimizeOSMO(target_geo, proj_geo, options):
    from ..projector.Projector3DParallel import Projector3DParallel

    A = projectorconstructor(target_geo, proj_geo)
    if (getattr(options, "engine", "device") == "host" or not isinstance(A, Projector3DParallel)
            or options.bit_depth is not None):
        return _osmo_host(target_geo, proj_geo, options, A)
    dev = A.device
    plan = A.plan
    ws = Workspace(dev)
    vs, ss = plan.shape_vol, plan.shape_sino
    mask = torch.as_tensor(metrics.region_mask(target_geo).reshape(vs), device=dev)
    n_iter = options.n_iter
    err_log = torch.full((max(n_iter, 1),), float("nan"), dtype=torch.float32, device=dev)
    counter = torch.zeros(1, dtype=torch.int32, device=dev)
    ver, xmax, bmax = ws.scalar(), ws.scalar(), ws.scalar()
    tgt = torch.as_tensor(np.ascontiguousarray(target_geo.array, dtype=np.float64), device=dev)
    xm = udata.filterTargetOSMO_t(tgt, options.filter).to(torch.float32).reshape(vs).contiguous()
    b = plan.forward(xm).clamp_(min=0)
    x = plan.backward_ref(b)
    ws.max(x, xmax)
    ws.scale(x, xmax)
    ws.ver(x, mask, ver)
    ws.append(ver, err_log, counter)
    inh = float(options.inhibition)

    def half(gel):
        ws.osmo_model(xm, x, None, mask, gel, options.d_h if gel else options.d_l)
        plan.forward(xm, b)
        ws.max(b, bmax)
        ws.scale(b, bmax, floor=inh)
        plan.backward_ref(b, x)
        ws.max(x, xmax)
        ws.scale(x, xmax, floor=0.0)

    def step():
        half(False)
        half(True)
        ws.ver(x, mask, ver)
        ws.append(ver, err_log, counter)

    st = torch.cuda.current_stream(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    done = 0
    if options.exit_param is None and n_iter > 2:
        gr = capture(step, dev)
        ev0.record(st)
        for _ in range(1, n_iter):
            gr.replay()
        ev1.record(st)
        done = n_iter - 1
    else:
        ev0.record(st)
        for _ in range(1, n_iter):
            step()
            done += 1
            if options.exit_param is not None and float(ver.item()) <= options.exit_param:
                break
        ev1.record(st)
    err = err_log.double().cpu().numpy()
    # device time per iteration of the loop (CUDA events on the engine's stream)
    options.device_iteration_ms = ev0.elapsed_time(ev1) / done if done else None
    err = np.where(np.arange(err.size) < int(counter.item()), err, np.nan)
    return (geometry.Sinogram(b.double().cpu().numpy(), proj_geo, options),
            geometry.Reconstruction(x.double().cpu().numpy(), proj_geo, options), err)
