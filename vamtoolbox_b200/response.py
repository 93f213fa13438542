"""Material response model: the reference's ``vamtoolbox.response.ResponseModel``.

Same constructor and methods as vamtoolbox/response.py:12-399 (generalised
logistic / linear / identity / freeform forms, analytical or 512-point
interpolation evaluation).  ``device_tables`` exposes the interpolation
tables to the fused BCLP kernel (vam_bclp_dose_pass), which evaluates map and
dmap/df with np.interp semantics (nearest-value extrapolation); analytical
generalised-logistic, linear and identity models are evaluated by the same
kernel in closed form, in float64 per voxel.
"""
from __future__ import annotations

import warnings

import numpy as np


class ResponseModel:
    _default_gen_log_fun = {"A": 0, "K": 1, "B": 25, "M": 0.5, "nu": 1}
    _default_linear = {"M": 1, "C": 0}
    _default_interpolation = {"interp_min": 0, "interp_max": 1, "n_pts": 512}

    def __init__(self, type="interpolation", form="gen_log_fun", **kwargs):
        self.type, self.form = type, form
        self._tables = {}
        if type == "analytical":
            if form == "gen_log_fun":
                self.map, self.dmapdf, self.map_inv = self._map_glf, self._dmapdf_glf, self._map_inv_glf
                self.params = dict(self._default_gen_log_fun)
            elif form == "linear":
                self.map, self.dmapdf, self.map_inv = self._map_lin, self._dmapdf_lin, self._map_inv_lin
                self.params = dict(self._default_linear)
            elif form == "identity":
                self.map, self.dmapdf, self.map_inv = self._map_id, self._dmapdf_id, self._map_inv_id
                self.params = {}
            else:
                raise Exception("Form: Other analytical functions are not supported yet.")
            self.params.update(kwargs)
        elif type == "interpolation":
            self.map, self.dmapdf, self.map_inv = self._map_interp, self._dmapdf_interp, self._map_inv_interp
            self.params = dict(self._default_interpolation)
            if form in ("gen_log_fun", "linear", "identity"):
                base = {"gen_log_fun": self._default_gen_log_fun, "linear": self._default_linear, "identity": {}}[form]
                self.params.update(base)
                self.params.update(kwargs)
                self.interp_f_0 = np.linspace(self.params["interp_min"], self.params["interp_max"], self.params["n_pts"])
                fm = {"gen_log_fun": (self._map_glf, self._dmapdf_glf), "linear": (self._map_lin, self._dmapdf_lin),
                      "identity": (self._map_id, self._dmapdf_id)}[form]
                self.interp_map_0 = fm[0](self.interp_f_0)
                self.interp_dmapdf_0 = fm[1](self.interp_f_0)
            elif form == "freeform":
                self.interp_f_0 = kwargs.get("interp_f_0")
                self.interp_map_0 = kwargs.get("interp_map_0")
                if self.interp_f_0.ndim > 1 or self.interp_map_0.ndim > 1:
                    raise Exception('Imported data for material response curve should be 1D. Check "interp_f_0" and "interp_map_0".')
                if self.interp_f_0.shape != self.interp_map_0.shape:
                    raise Exception('Size mismatch between "interp_f_0" and "interp_map_0".')
                self.interp_dmapdf_0 = np.diff(self.interp_map_0, n=1, append=(
                    self.interp_map_0[-1] + (self.interp_map_0[-1] - self.interp_map_0[-2])))
            else:
                raise Exception("Other interpolation functions are not supported yet.")
        else:
            raise Exception('Mapping type ("type") should be either "analytical" or "interpolation".')

    # generalised logistic function (Richards' curve)
    def _map_glf(self, f):
        p = self.params
        self.cached_exp = np.exp(-p["B"] * (f - p["M"]))
        self.cached_map = p["A"] + (p["K"] - p["A"]) / (1 + self.cached_exp) ** (1 / p["nu"])
        return self.cached_map

    def _dmapdf_glf(self, f, use_cached_result=False):
        p = self.params
        c1 = (1 / (p["K"] - p["A"])) ** p["nu"]
        c2 = p["B"] / p["nu"]
        if use_cached_result:
            c3 = (self.cached_map - p["A"]) ** (p["nu"] + 1)
            ex = self.cached_exp
        else:
            c3 = (self._map_glf(f) - p["A"]) ** (p["nu"] + 1)
            ex = np.exp(-p["B"] * (f - p["M"]))
        self.cached_dmapdf = c1 * c2 * c3 * ex
        return self.cached_dmapdf

    def _map_inv_glf(self, mapped):
        p = self.params
        num = -np.log(((p["K"] - p["A"]) / (mapped - p["A"])) ** p["nu"] - 1)
        return num / p["B"] + p["M"]

    def _map_lin(self, f):
        self.cached_map = self.params["M"] * f + self.params["C"]
        return self.cached_map

    def _dmapdf_lin(self, f, use_cached_result=False):
        return np.ones_like(f) * self.params["M"]

    def _map_inv_lin(self, mapped):
        return (mapped - self.params["C"]) / self.params["M"]

    def _map_id(self, f):
        self.cached_map = f
        return f

    def _dmapdf_id(self, f, use_cached_result=False):
        return np.ones_like(f)

    def _map_inv_id(self, mapped):
        return mapped

    def _map_interp(self, f):
        return np.interp(f, self.interp_f_0, self.interp_map_0, left=self.interp_map_0[0], right=self.interp_map_0[-1])

    def _dmapdf_interp(self, f):
        return np.interp(f, self.interp_f_0, self.interp_dmapdf_0, left=self.interp_dmapdf_0[0],
                         right=self.interp_dmapdf_0[-1])

    def _map_inv_interp(self, mapped):
        return np.interp(mapped, self.interp_map_0, self.interp_f_0, left=self.interp_f_0[0], right=self.interp_f_0[-1])

    def checkResponseTarget(self, f_T):
        """Reachability / finiteness check of the response target (response.py:363-396)."""
        f_T = np.asarray(f_T)
        lo, hi = np.amin(f_T), np.amax(f_T)
        ok = True
        if self.form == "gen_log_fun" and hi > self.params["K"]:
            warnings.warn("Maximum response target is greater than right asymptotic value of response function.")
            ok = False
        m0 = self.map(0)
        if (lo < m0) and ~(np.isclose(lo, m0, atol=0.01 * hi)):
            warnings.warn("Minimum response target is lower than response at zero optical dose.")
            ok = False
        if np.isinf(f_T).any():
            warnings.warn("Response target contains infinite value(s).")
            ok = False
        if np.isnan(f_T).any():
            warnings.warn("Response target contains nan value(s).")
            ok = False
        return ok

    # ------------------------------------------------------------------
    def has_uniform_table(self):
        if self.type != "interpolation":
            return False
        f = np.asarray(self.interp_f_0, dtype=np.float64)
        if f.size < 2:
            return False
        d = np.diff(f)
        return bool(np.all(d > 0) and np.allclose(d, d[0], rtol=1e-9, atol=0))

    def has_device_form(self):
        """True when the fused BCLP dose pass evaluates this model on the device: an interpolation
        table with strictly increasing sample points (np.interp's requirement; its bins are found by a
        search seeded as if uniform), or an analytical generalised-logistic / linear / identity form
        in closed form."""
        if self.type == "analytical":
            return self.form in ("gen_log_fun", "linear", "identity")
        f = np.asarray(self.interp_f_0, dtype=np.float64)
        return bool(f.size >= 2 and np.all(np.diff(f) > 0) and np.asarray(self.interp_map_0).shape == f.shape)

    # -- device forms of the set-up steps (torch float64, same values as the numpy methods) -------
    def device_map_inv_ok(self):
        """map_inv has a device form: the closed forms, or np.interp on an increasing map table."""
        if self.type == "analytical":
            return self.form in ("gen_log_fun", "linear", "identity")
        m = np.asarray(self.interp_map_0, dtype=np.float64)
        return bool(m.size >= 2 and np.all(np.diff(m) > 0))

    def map_inv_t(self, mapped):
        """map_inv of a float64 CUDA tensor (response.py:220-237, 281-290)."""
        import torch

        if self.type == "analytical":
            p = self.params
            if self.form == "gen_log_fun":
                num = -torch.log(((p["K"] - p["A"]) / (mapped - p["A"])) ** p["nu"] - 1)
                return num / p["B"] + p["M"]
            if self.form == "linear":
                return (mapped - p["C"]) / p["M"]
            return mapped.clone()
        return _interp_t(mapped, torch.as_tensor(np.asarray(self.interp_map_0, np.float64), device=mapped.device),
                         torch.as_tensor(np.asarray(self.interp_f_0, np.float64), device=mapped.device))

    def checkResponseTarget_t(self, f_T):
        """checkResponseTarget of a CUDA tensor: the four reductions on the device, one read-back."""
        import torch

        lo, hi = torch.aminmax(f_T)
        flags = torch.stack([lo, hi, torch.isinf(f_T).any().to(f_T.dtype), torch.isnan(f_T).any().to(f_T.dtype)]).cpu()
        lo, hi, has_inf, has_nan = (float(v) for v in flags)
        ok = True
        if self.form == "gen_log_fun" and hi > self.params["K"]:
            warnings.warn("Maximum response target is greater than right asymptotic value of response function.")
            ok = False
        m0 = self.map(0)
        if (lo < m0) and ~(np.isclose(lo, m0, atol=0.01 * hi)):
            warnings.warn("Minimum response target is lower than response at zero optical dose.")
            ok = False
        if has_inf:
            warnings.warn("Response target contains infinite value(s).")
            ok = False
        if has_nan:
            warnings.warn("Response target contains nan value(s).")
            ok = False
        return ok

    def device_tables(self, device):
        """float32 (f, map, dmap) tables on `device` for the fused BCLP kernel."""
        import torch

        key = str(device)
        if key not in self._tables:
            mk = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float32), device=device).contiguous()
            f = np.asarray(self.interp_f_0, dtype=np.float64)
            self._tables[key] = (mk(f), mk(self.interp_map_0), mk(self.interp_dmapdf_0),
                                 float(np.float32(f[0])), float((f.size - 1) / (f[-1] - f[0])))
        return self._tables[key]

    def _no_display(self, name):
        import logging

        logging.getLogger(__name__).warning("ResponseModel.%s(): no display in this package", name)

    def plotMap(self, *args, **kwargs):
        """The reference plots the response curve with matplotlib (response.py:294-339); headless here:
        logs and returns (the curve is ``map`` over a dose range)."""
        self._no_display("plotMap")

    def plotDmapDf(self, *args, **kwargs):
        """Headless counterpart of the reference's derivative plot: logs and returns."""
        self._no_display("plotDmapDf")

    def plotMapInv(self, *args, **kwargs):
        """Headless counterpart of the reference's inverse-map plot (response.py:340-): logs and returns."""
        self._no_display("plotMapInv")

    def __repr__(self):
        return str(self.params)


def _interp_t(x, xp, fp):
    """np.interp(x, xp, fp) with nearest-value extrapolation (left = fp[0], right = fp[-1]) for an
    increasing xp, on CUDA float64 tensors: bin by searchsorted, then fp[j] + slope (x - xp[j])."""
    import torch

    n = xp.numel()
    j = (torch.searchsorted(xp, x, right=True) - 1).clamp_(0, n - 2)
    x0, x1, y0, y1 = xp[j], xp[j + 1], fp[j], fp[j + 1]
    y = (y1 - y0) / (x1 - x0) * (x - x0) + y0
    y = torch.where(x == x0, y0, y)
    y = torch.where(x < xp[0], fp[0], y)
    y = torch.where(x >= xp[-1], fp[-1], y)
    return torch.where(torch.isnan(x), x, y)
