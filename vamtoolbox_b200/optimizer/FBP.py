"""Filtered backprojection (vamtoolbox/optimizer/FBP.py): one forward, filter, one backward."""
from __future__ import annotations

import numpy as np
import torch

from .. import geometry, metrics
from ..projectorconstructor import projectorconstructor
from ..util import data as udata


def minimizeFBP(target_geo, proj_geo, options):
    A = projectorconstructor(target_geo, proj_geo)
    err = np.full(options.n_iter, np.nan)
    if hasattr(getattr(A, "plan", None), "backward_ref"):  # parallel beam: cuFFT filter on the device
        b = udata.filterSinogram_t(A.forward_t(target_geo.array), options.filter).double().cpu().numpy()
    else:
        b = udata.filterSinogram(A.forward(target_geo.array), options.filter)
    if getattr(options, "offset", False):
        b = b + np.broadcast_to(np.abs(np.min(b, axis=0)), b.shape)
    else:
        b = np.clip(b, a_min=0, a_max=None)
    b = b / np.max(b)
    if options.bit_depth is not None:
        b = udata.discretize(b, options.bit_depth, [0.0, np.max(b)])
    x = A.backward(b)
    x = x / np.max(x)
    err[0] = metrics.calcVER(target_geo, x)
    return geometry.Sinogram(b, proj_geo, options), geometry.Reconstruction(x, proj_geo, options), err
