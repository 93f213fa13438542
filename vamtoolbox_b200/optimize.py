"""Optimizer front end: the reference's ``vamtoolbox.optimize`` (vamtoolbox/optimize.py:1-217).

``Options`` takes the reference's keyword arguments and defaults per method
(FBP, CAL, PM, OSMO, BCLP).  Unlike the reference, each instance starts from
fresh defaults: the reference's class-level default dicts are updated by
every construction (optimize.py:119-126), so keyword arguments leak from one
Options object to the next in a process; that leak is not reproduced.

Extra keyword:
    engine : "device" (default) runs the iteration bodies as fused sm_100a
             kernels on device-resident arrays, BCLP / CAL / OSMO iterations
             captured once in a CUDA graph and replayed;
             "host" runs the reference's numpy loop and calls the projector
             per step with host arrays (the plain per-call GPU path).
"""
from __future__ import annotations

from . import geometry


class Options:
    _default_FBP = {"offset": False}
    _default_CAL = {"learning_rate": 0.01, "momentum": 0, "positivity": 0, "sigmoid": 0.01}
    _default_PM = {"rho_1": 1, "rho_2": 1, "p": 1}
    _default_OSMO = {"inhibition": 0}
    _default_BCLP = {"response_model": "default", "eps": 0.1, "weight": 1, "p": 2, "q": 1, "learning_rate": 0.01,
                     "optim_alg": "grad_des", "g0": None}

    def __init__(self, method="CAL", n_iter=50, d_h=0.8, d_l=0.7, filter="ram-lak", units="normalized", blb=0,
                 bub=None, **kwargs):
        self.method = method
        self.n_iter = n_iter
        self.d_h = d_h
        self.d_l = d_l
        self.filter = filter
        self.units = units
        self.blb = blb
        self.bub = bub
        self.__dict__.update(kwargs)
        self.verbose = self.__dict__.get("verbose", False)
        self.save_img_path = self.__dict__.get("save_img_path", None)
        self.bit_depth = self.__dict__.get("bit_depth", None)
        self.exit_param = self.__dict__.get("exit_param", None)
        self.engine = self.__dict__.get("engine", "device")
        if self.engine not in ("device", "host"):
            raise ValueError("engine must be 'device' or 'host'")
        d = {}
        for name in ("FBP", "CAL", "PM", "OSMO", "BCLP"):
            dd = dict(getattr(self, "_default_" + name))
            dd.update({k: v for k, v in kwargs.items() if k in dd})
            d[name] = dd
        if method == "FBP":
            self.offset = d["FBP"]["offset"]
        if method == "CAL":
            for k in ("learning_rate", "momentum", "positivity", "sigmoid"):
                setattr(self, k, d["CAL"][k])
        if method == "PM":
            for k in ("rho_1", "rho_2", "p"):
                setattr(self, k, d["PM"][k])
        if method == "OSMO":
            self.inhibition = d["OSMO"]["inhibition"]
        if method == "BCLP":
            from .response import ResponseModel

            rm = d["BCLP"]["response_model"]
            self.response_model = ResponseModel() if (isinstance(rm, str) and rm == "default") else rm
            for k in ("eps", "weight", "p", "q", "learning_rate", "optim_alg", "g0"):
                setattr(self, k, d["BCLP"][k])
            self.test_alternate_handling = self.__dict__.get("test_alternate_handling", False)

    def __str__(self):
        return str(self.__dict__)


def optimize(target_geo, proj_geo, options, output="packaged"):
    """Run the optimizer named by ``options.method`` (optimize.py:174-217).

    Returns (Sinogram, Reconstruction, error) like the reference; BCLP also
    accepts output="full" / "components".
    """
    from .optimizer import BCLP, CAL, FBP, OSMO, PM

    if options.units != "normalized" or proj_geo.absorption_coeff is not None:
        proj_geo.calcAbsorptionMask(target_geo)
    if options.method == "FBP":
        return FBP.minimizeFBP(target_geo, proj_geo, options)
    if options.method == "CAL":
        return CAL.minimizeCAL(target_geo, proj_geo, options)
    if options.method == "PM":
        return PM.minimizePM(target_geo, proj_geo, options)
    if options.method == "OSMO":
        return OSMO.minimizeOSMO(target_geo, proj_geo, options)
    if options.method == "BCLP":
        return BCLP.minimizeBCLP(target_geo, proj_geo, options, output)
    raise ValueError(f"unknown method {options.method!r}")


__all__ = ["Options", "optimize", "geometry"]
