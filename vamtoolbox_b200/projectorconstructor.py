"""Projector factory: the reference's ``projectorconstructor`` (vamtoolbox/projectorconstructor.py:21-165).

Keeps the reference's dispatch keys (``ray_type``, ``attenuation_field`` /
``insert``, ``absorption_coeff``, ``n_dim``) and side effects (an insert
becomes infinite attenuation, a zero-dose region becomes
``proj_geo.zero_dose_sino``), but every parallel-beam branch -- CPU or
``CUDA=True``, with or without attenuation, 2-D or 3-D -- returns the same
sm_100a projector, including the ``CUDA=True`` + attenuation combination the
reference rejects with NotImplementedError (:89-97).
"""
from __future__ import annotations

from typing import Protocol

import numpy as np


class Projector(Protocol):
    """Protocol of the projector objects (projectorconstructor.py:13-18)."""

    def forward(self, x): ...

    def backward(self, b): ...


class CALopticalparams:
    def __init__(self, *args, **kwargs):
        raise NotImplementedError


def _astra_model(proj_geo):
    """Inclined rays (laminography) exist only in the reference's ASTRA path
    (Projector3DParallelCUDA.py:27-38), so they select the vector-geometry
    projector; ``parallel_model="astra"`` selects it for vertical rays too."""
    incl = getattr(proj_geo, "inclination_angle", None)
    return (incl is not None and incl != 0) or getattr(proj_geo, "parallel_model", None) == "astra"


def projectorconstructor(target_geo, proj_geo, optical_params=None, **projector_kwargs):
    """Build the projector for ``target_geo`` / ``proj_geo``.

    Extra keyword arguments go to the projector (e.g. ``absorption="ray"``
    or ``device=...`` for the parallel-beam projector).
    """
    if getattr(target_geo, "insert", None) is not None:
        ins = np.asarray(target_geo.insert) == 1
        if proj_geo.attenuation_field is not None:
            proj_geo.attenuation_field[ins] = np.inf
        else:
            proj_geo.attenuation_field = np.where(ins, np.inf, 0)

    if proj_geo.ray_type == "algebraic":
        from .projector.pyTorchAlgebraicPropagation import PyTorchAlgebraicPropagator

        A = PyTorchAlgebraicPropagator(target_geo, proj_geo, **projector_kwargs)
    elif proj_geo.ray_type == "ray_trace":
        from .projector.pyTorchRayTrace import PyTorchRayTracingPropagator

        A = PyTorchRayTracingPropagator(target_geo, proj_geo, **projector_kwargs)
    elif proj_geo.ray_type in ("parallel", None):
        if target_geo.n_dim == 2 and getattr(proj_geo, "parallel_model", None) == "astra":
            from .projector.Projector2DParallelCUDA import Projector2DParallelCUDAAstra

            A = Projector2DParallelCUDAAstra(target_geo, proj_geo, **projector_kwargs)
        elif target_geo.n_dim == 2:
            from .projector.Projector2DParallel import Projector2DParallel

            A = Projector2DParallel(target_geo, proj_geo, **projector_kwargs)
        elif _astra_model(proj_geo):
            from .projector.Projector3DParallelCUDA import Projector3DParallelCUDAAstra

            if getattr(proj_geo, "attenuation_field", None) is not None:
                raise NotImplementedError("3D attenuation CUDA projector not yet implemented.")
            A = Projector3DParallelCUDAAstra(target_geo, proj_geo, **projector_kwargs)
        else:
            from .projector.Projector3DParallel import Projector3DParallel

            A = Projector3DParallel(target_geo, proj_geo, **projector_kwargs)
    else:
        raise NotImplementedError(f"ray_type {proj_geo.ray_type!r} is not supported")

    if getattr(target_geo, "zero_dose", None) is not None:
        proj_geo.calcZeroDoseSinogram(A, target_geo)
    return A
