"""Propagation-medium models: the reference's ``vamtoolbox.medium`` interface.

IndexModel / AttenuationModel / AbsorptionModel keep the reference's
constructor arguments and query methods (vamtoolbox/medium.py:13-1002):
``n(x)``, ``grad_n(x)``, ``alpha(x)`` on [N, 3] position tensors, the
presampled-field path with central-difference gradients, and the analytic
forms (homogeneous, Luneburg lens, homogeneous cylinder / ball).  On top of
that each model describes itself to the ray-tracing kernel
(:meth:`IndexModel.kernel_fields`, :meth:`AttenuationModel.kernel_fields`),
which samples the fields itself; ``grid_sample`` is used here only for host
queries and setup, never inside the ray loop.
"""
from __future__ import annotations

import logging

import numpy as np
import torch

from . import _lib


def _default_device():
    return torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else torch.device("cpu")


class MediumModel:
    """Coordinate grid shared by the medium models (medium.py:13-273)."""

    def __init__(self, coord_vec, device=None):
        self.device = torch.device(device) if device is not None else _default_device()
        self.xv = torch.as_tensor(np.asarray(coord_vec[0], dtype=np.float64), device=self.device)
        self.yv = torch.as_tensor(np.asarray(coord_vec[1], dtype=np.float64), device=self.device)
        self.zv = torch.as_tensor(np.asarray(coord_vec[2], dtype=np.float64), device=self.device)
        self.coord_vec = [np.asarray(c, dtype=np.float64) for c in coord_vec]
        self.xg, self.yg, self.zg = torch.meshgrid(self.xv, self.yv, self.zv, indexing="ij")
        self.xv_yv_zv_max = torch.stack([self.xv.max(), self.yv.max(), self.zv.max()])
        self.xv_yv_zv_min = torch.stack([self.xv.min(), self.yv.min(), self.zv.min()])
        if self.zv.numel() == 1:
            self.voxel_size = torch.stack([self.xv[1] - self.xv[0], self.yv[1] - self.yv[0],
                                           torch.tensor(float("inf"), dtype=torch.float64, device=self.device)])
        else:
            self.voxel_size = torch.stack([self.xv[1] - self.xv[0], self.yv[1] - self.yv[0], self.zv[1] - self.zv[0]])
        self.grid_span = self.xv_yv_zv_max - self.xv_yv_zv_min
        self.position_normalization_factor = 2.0 / self.grid_span
        if torch.isinf(self.position_normalization_factor[2]):
            self.position_normalization_factor[2] = 0.0
        self.presampled_scalar_field_3D = None
        self.presampled_vector_field_4D = None
        self.interpolation_padding_mode = "border"

    @property
    def shape(self):
        return tuple(self.xg.shape)

    def getPositionVectorsAtGridPoints(self):
        return torch.vstack((self.xg.ravel(), self.yg.ravel(), self.zg.ravel())).T

    def normalizePosition(self, x):
        return x * self.position_normalization_factor

    def _field5d(self, f3):
        return torch.permute(f3, (2, 1, 0))[None, None]

    def _scalar_field_interp(self, x):
        g = self.normalizePosition(x.to(torch.float64))
        out = torch.nn.functional.grid_sample(self._field5d(self.presampled_scalar_field_3D.to(torch.float64)),
                                              g[None, None, None], mode="bilinear",
                                              padding_mode=self.interpolation_padding_mode, align_corners=True)
        return out[0, 0, 0, 0, :]

    def _vector_field_interp(self, x):
        g = self.normalizePosition(x.to(torch.float64))
        f = torch.permute(self.presampled_vector_field_4D.to(torch.float64), (3, 2, 1, 0))[None]
        out = torch.nn.functional.grid_sample(f, g[None, None, None], mode="bilinear",
                                              padding_mode=self.interpolation_padding_mode, align_corners=True)
        return out[0, :, 0, 0, :].T

    @staticmethod
    def centralFiniteDifference(field, voxel_size):
        """Central differences with zero boundary faces (medium.py:224-273)."""
        f = field
        vs = [float(v) for v in voxel_size]
        d = torch.zeros(f.shape + (3,), dtype=f.dtype, device=f.device)
        d[1:-1, :, :, 0] = (f[2:] - f[:-2]) / (2 * vs[0])
        d[:, 1:-1, :, 1] = (f[:, 2:] - f[:, :-2]) / (2 * vs[1])
        if f.shape[2] > 1 and np.isfinite(vs[2]):
            d[:, :, 1:-1, 2] = (f[:, :, 2:] - f[:, :, :-2]) / (2 * vs[2])
        return d

    def _fractional_radius(self, R):
        spans = [(np.amax(c) - np.amin(c)) / 2 for c in self.coord_vec]
        return R * (min(spans[0], spans[1]) if self.coord_vec[2].size == 1 else min(spans))


def _no_display(obj, name):
    """The reference draws these with matplotlib; this package has no display: log that nothing is drawn
    and return, so a script runs to the end headless (the fields are the model's presampled arrays)."""
    logging.getLogger(__name__).warning("%s.%s(): no display in this package", type(obj).__name__, name)


class IndexModel(MediumModel):
    """Refractive index n(x) and its gradient (medium.py:276-473)."""

    _default_analytical = {"R": 1.0, "length_unit_of_R": "fractional_domain_radius", "p": 2.0, "n_sur": 1.0}
    _default_interpolation = {"interpolation_padding_mode": "border"}

    def __init__(self, coord_vec, type="analytical", form="homogeneous", device=None, **kwargs):
        super().__init__(coord_vec, device)
        self.logger = logging.getLogger(__name__)
        self.type, self.form = type, form
        self.params = dict(self._default_analytical)
        self.params.update(self._default_interpolation)
        self.params.update(kwargs)
        if self.params["length_unit_of_R"] == "fractional_domain_radius":
            self.params["R_physical"] = self._fractional_radius(self.params["R"])
        elif self.params["length_unit_of_R"] == "physical_coordinate":
            self.params["R_physical"] = self.params["R"]
        else:
            raise Exception('"length_unit" should be either "fractional_domain_radius" or "physical_coordinate"')
        forms = {"homogeneous": (self._n_homo, self._grad_n_homo), "luneburg_lens": (self._n_lune, self._grad_n_lune)}
        if form in ("maxwell_lens", "eaton_lens"):
            raise Exception("To be implemented.")
        if type == "analytical":
            if form not in forms:
                raise Exception("Form: Other analytical functions are not supported yet.")
            self.n, self.grad_n = forms[form]
        elif type == "interpolation":
            self.n, self.grad_n = self._scalar_field_interp, self._vector_field_interp
            self.interpolation_padding_mode = self.params["interpolation_padding_mode"]
            x = self.getPositionVectorsAtGridPoints()
            if form in forms:
                nf, gf = forms[form]
                self.presampled_scalar_field_3D = nf(x).reshape(self.shape)
                self.presampled_vector_field_4D = gf(x).reshape(self.shape + (3,))
            elif form == "freeform":
                n_x = self.params.get("n_x")
                g_x = self.params.get("grad_n_x")
                self.presampled_scalar_field_3D = torch.as_tensor(n_x, device=self.device)
                self.presampled_vector_field_4D = None if g_x is None else torch.as_tensor(g_x, device=self.device)
            else:
                raise Exception("Other interpolation functions are not supported yet.")
            f3 = self.presampled_scalar_field_3D
            if f3.ndim <= 2:
                raise Exception('Imported scalar field ("n_x" or "alpha_x") should be 3D (even in 2D the thrid dim should have size 1).')
            if tuple(f3.shape) != self.shape:
                raise Exception(f"Size mismatch between the constructed coordinate grid ({self.shape}) and imported scalar field ({tuple(f3.shape)}).")
            if self.presampled_vector_field_4D is None:
                self.presampled_vector_field_4D = self.centralFiniteDifference(f3, self.voxel_size)
            elif tuple(self.presampled_vector_field_4D.shape) != self.shape + (3,):
                raise Exception("Index gradient field should have extactly one more dimension (of size 3) than index field.")
        else:
            raise Exception('"type" should be either "analytical" or "interpolation".')

    def _n_homo(self, x):
        return self.params["n_sur"] * torch.ones_like(x[:, 0])

    def _grad_n_homo(self, x):
        return torch.zeros_like(x)

    def _n_lune(self, x=None, r_known=None):
        r = torch.sqrt(x[:, 0] ** 2 + x[:, 1] ** 2 + x[:, 2] ** 2) if r_known is None else r_known
        n = torch.ones_like(r)
        R, p, n0 = self.params["R_physical"], self.params["p"], self.params["n_sur"]
        inside = r < R
        n[inside] = n0 * (2 - (r[inside] / R) ** p) ** (1 / p)
        if n0 != 1.0:
            n[~inside] = n0
        return n

    def _grad_n_lune(self, x):
        r = torch.sqrt(x[:, 0] ** 2 + x[:, 1] ** 2 + x[:, 2] ** 2)
        n = self._n_lune(r_known=r)
        g = torch.zeros_like(x)
        R, p, n0 = self.params["R_physical"], self.params["p"], self.params["n_sur"]
        inside = r < R
        g[inside, :] = -((n0 / R) ** p) * ((n[inside] ** (1 - p)) * (r[inside] ** (p - 2)))[:, None] * x[inside, :]
        return g

    def kernel_fields(self):
        """(kind, n_sur, R, p, n_grid float32, grad_grid float32) for the ray kernel."""
        if self.type == "analytical" and self.form == "homogeneous":
            return _lib.INDEX_HOMOGENEOUS, float(self.params["n_sur"]), 0.0, 0.0, None, None
        if self.type == "analytical" and self.form == "luneburg_lens":
            return (_lib.INDEX_LUNEBURG, float(self.params["n_sur"]), float(self.params["R_physical"]),
                    float(self.params["p"]), None, None)
        n = self.presampled_scalar_field_3D.to(device=self.device, dtype=torch.float32).contiguous()
        g = self.presampled_vector_field_4D.to(device=self.device, dtype=torch.float32).contiguous()
        return _lib.INDEX_GRID, 1.0, 0.0, 0.0, n, g


class AttenuationModel(MediumModel):
    """Attenuation (or absorption) coefficient alpha(x) (medium.py:753-915)."""

    _default_analytical = {"R": 1.0, "length_unit_of_R": "fractional_domain_radius", "alpha_internal": 1e-3}
    _default_interpolation = {"interpolation_padding_mode": "zeros"}

    def __init__(self, coord_vec, type="analytical", form="homogeneous_cylinder", device=None, **kwargs):
        super().__init__(coord_vec, device)
        self.logger = logging.getLogger(__name__)
        self.type, self.form = type, form
        self.params = dict(self._default_analytical)
        self.params.update(self._default_interpolation)
        self.params.update(kwargs)
        if self.params["length_unit_of_R"] == "fractional_domain_radius":
            self.params["R_physical"] = self._fractional_radius(self.params["R"])
        elif self.params["length_unit_of_R"] == "physical_coordinate":
            self.params["R_physical"] = self.params["R"]
        else:
            raise Exception('"length_unit" should be either "fractional_domain_radius" or "physical_coordinate"')
        forms = {"homogeneous_cylinder": self._alpha_homo_cylinder, "homogeneous_ball": self._alpha_homo_ball}
        if type == "analytical":
            if form not in forms:
                raise Exception("Form: Other analytical functions are not supported yet.")
            self.alpha = forms[form]
        elif type == "interpolation":
            self.alpha = self._scalar_field_interp
            self.interpolation_padding_mode = self.params["interpolation_padding_mode"]
            if form in forms:
                self.presampled_scalar_field_3D = forms[form](self.getPositionVectorsAtGridPoints()).reshape(self.shape)
            elif form == "freeform":
                self.presampled_scalar_field_3D = torch.as_tensor(self.params.get("alpha_x"), device=self.device)
            else:
                raise Exception("Other interpolation functions are not supported yet.")
            if tuple(self.presampled_scalar_field_3D.shape) != self.shape:
                raise Exception("Size mismatch between the constructed coordinate grid and imported scalar field.")
        else:
            raise Exception('"type" should be either "analytical" or "interpolation".')

    def _alpha_homo_cylinder(self, x):
        r = torch.linalg.norm(x[:, 0:2], dim=1)
        a = torch.zeros_like(r)
        a[r < self.params["R_physical"]] = self.params["alpha_internal"]
        return a

    def _alpha_homo_ball(self, x):
        r = torch.linalg.norm(x, dim=1)
        a = torch.zeros_like(r)
        a[r < self.params["R_physical"]] = self.params["alpha_internal"]
        return a

    def kernel_fields(self):
        """(kind, value, R, grid float32) for the ray kernel's attenuation sampling."""
        if self.type == "analytical":
            kind = _lib.ALPHA_CYLINDER if self.form == "homogeneous_cylinder" else _lib.ALPHA_BALL
            return kind, float(self.params["alpha_internal"]), float(self.params["R_physical"]), None
        g = self.presampled_scalar_field_3D.to(device=self.device, dtype=torch.float32).contiguous()
        return _lib.ALPHA_GRID, 0.0, 0.0, g

    def alpha_at_grid(self):
        """alpha at the grid points, float32 [nX, nY, nZ] (pyTorchRayTrace.py:458-462)."""
        if self.type == "interpolation":
            return self.presampled_scalar_field_3D.to(dtype=torch.float32).contiguous()
        return self.alpha(self.getPositionVectorsAtGridPoints()).reshape(self.shape).to(torch.float32).contiguous()


def _headless(name):
    def method(self, *args, **kwargs):
        _no_display(self, name)

    method.__name__ = name
    method.__doc__ = "The reference's plot of the field (medium.py); headless here: logs and returns."
    return method


# the reference's plotting methods (medium.py:570-751, 918-990), headless
for _cls, _names in ((IndexModel, ("plotIndex", "plotGradNMag", "plotRandomlySampledIndex", "plotIndexAtPosition")),
                     (AttenuationModel, ("plotAlpha", "plotRandomlySampledAlpha", "plotAlphaAtPosition"))):
    for _n in _names:
        setattr(_cls, _n, _headless(_n))


class AbsorptionModel(AttenuationModel):
    """Alias of AttenuationModel (medium.py:993-996)."""


class ScatteringModel(AttenuationModel):
    """Reserved, as in the reference (medium.py:999-1002)."""
