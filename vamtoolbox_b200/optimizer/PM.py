"""Penalty minimisation with L-BFGS-B (vamtoolbox/optimizer/PM.py).

The quasi-Newton driver stays scipy's L-BFGS-B on the host (as in the
reference); each loss / gradient evaluation runs the projector and the
penalty terms on the GPU and returns float64 host values to scipy.
"""
from __future__ import annotations

import time

import numpy as np
import torch
from scipy import optimize as spo

from .. import geometry, metrics
from ..projectorconstructor import projectorconstructor
from ..util import data as udata


class LogError:
    def __init__(self, options):
        self.options = options
        self.curr_iter = 0
        self.error_iter = 0
        self.loss = []
        self.error = np.full(options.n_iter + 1, np.nan)
        self.iter_times = np.zeros(options.n_iter + 1)
        self.t0 = time.perf_counter()

    def getIterTime(self, i):
        self.iter_times[i] = time.perf_counter() - self.t0


def minimizePM(target_geo, proj_geo, options):
    A = projectorconstructor(target_geo, proj_geo)
    dev = getattr(A, "device", torch.device("cuda"))
    core = torch.as_tensor(np.asarray(target_geo.gel_inds), device=dev)
    background = torch.as_tensor(np.asarray(target_geo.void_inds), device=dev)
    b0 = A.forward(target_geo.array)
    shape = b0.shape
    b0 = udata.filterSinogram(b0, options.filter)
    b0 = np.clip(b0, a_min=0, a_max=None)
    b0 = b0 / np.max(b0)
    log = LogError(options)
    x0 = A.backward(b0)
    log.error[0] = metrics.calcVER(target_geo, x0 / np.max(x0))
    log.iter_times[0] = time.perf_counter() - log.t0
    state = {}
    fac = np.pi / 180

    def regions(dose):
        V1 = core & ~(dose >= options.d_h)
        V2 = background & ~(dose <= options.d_l)
        return V1, V2

    def loss(bflat):
        if options.bit_depth is not None:
            bflat = udata.discretize(bflat, options.bit_depth, [0.0, np.max(bflat)])
        bt = torch.as_tensor(np.reshape(bflat, shape), device=dev, dtype=torch.float32)
        dose = A.backward(bt).reshape(core.shape).double() * fac
        state["dose"] = dose
        log.error_iter = metrics.calcVER(target_geo, dose)
        V1, V2 = regions(dose)
        integrand = (options.rho_1 * (dose - options.d_l) ** options.p * V2
                     + options.rho_2 * (options.d_h - dose) ** options.p * V1)
        v = float(integrand.sum())
        log.loss.append(v)
        return v

    def grad(bflat):
        dose = state["dose"]
        V1, V2 = regions(dose)
        gd = (options.rho_1 * V2.double() * options.p * (dose - options.d_l) ** (options.p - 1)
              - options.rho_2 * V1.double() * options.p * (options.d_h - dose) ** (options.p - 1))
        g = A.forward(gd.to(torch.float32).reshape(A.plan.shape_vol if hasattr(A, "plan") else gd.shape))
        g = g.double().cpu().numpy() if isinstance(g, torch.Tensor) else np.asarray(g)
        return np.reshape(g, -1) * fac

    def callback(_):
        log.getIterTime(log.curr_iter + 1)
        log.error[log.curr_iter + 1] = log.error_iter
        log.curr_iter += 1

    res = spo.minimize(fun=loss, x0=np.reshape(b0, -1), callback=callback, method="L-BFGS-B", jac=grad,
                       bounds=[(0, 1)] * b0.size,
                       options={"maxiter": options.n_iter, "ftol": 1e-12, "disp": False, "maxcor": 10, "maxls": 30})
    log.loss = np.array(log.loss)
    b_opt = np.reshape(res.x, shape)
    if options.bit_depth is not None:
        b_opt = udata.discretize(b_opt, options.bit_depth, [0.0, np.max(b_opt)])
    x_opt = A.backward(b_opt) * np.pi / 180
    return geometry.Sinogram(b_opt, proj_geo, options), geometry.Reconstruction(x_opt, proj_geo, options), log.error
