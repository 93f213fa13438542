"""Geometry data model: the reference's ``vamtoolbox.geometry`` interface.

Mirrors vamtoolbox/geometry.py (ProjectionGeometry :30-193, Volume / TargetGeometry
/ Sinogram / Reconstruction :196-659, loadVolume :662-679, getCircleMask /
getInds :682-733) so that user code written for the reference constructs the
same objects.  Arrays stay numpy on this side; the projectors move them to
the device.  ``rebinFanBeam`` (geometry.py:736-944) resamples on the GPU
(libvamcore vam_rebin_fan) from grid-search tables built here.
"""
from __future__ import annotations

import numpy as np

from .util import data as _data

_PROJ_KWARGS = (
    "projector_pixel_size", "absorption_coeff", "container_radius", "attenuation_field", "occlusion",
    "inclination_angle", "zero_dose_sino", "index_model", "attenuation_model", "absorption_model",
    "ray_trace_method", "eikonal_parametrization", "ray_trace_ode_solver", "ray_trace_ray_config",
    "tensor_dtype", "ray_density",
)


class ProjectionGeometry:
    """Projection geometry keyword bag (vamtoolbox/geometry.py:30-155).

    Parameters are the reference's: ``angles`` (degrees), ``ray_type``
    ("parallel", "ray_trace", "algebraic"), ``CUDA`` and the optional keywords
    listed in :data:`_PROJ_KWARGS`.  ``CUDA`` is accepted for compatibility;
    every projector of this package runs on the GPU.
    """

    def __init__(self, angles, ray_type="parallel", CUDA=False, **kwargs):
        self.angles = np.asarray(angles)
        self.n_angles = int(np.size(self.angles))
        self.ray_type = ray_type
        self.CUDA = CUDA
        for k in _PROJ_KWARGS:
            setattr(self, k, kwargs.get(k, None))
        self.loading_path_for_matrix = kwargs.get("loading_path_for_matrix", True)
        # "python" (default): the discretisation of the reference's Python projectors;
        # "astra": the vector-geometry model of its CUDA path (always used for inclined rays)
        self.parallel_model = kwargs.get("parallel_model", "python")
        self.absorption_mask = None

    def calcZeroDoseSinogram(self, A, target_geo):
        """Sinogram entries that would reach a zero-dose region (geometry.py:157-159)."""
        b = A.forward(target_geo.zero_dose)
        b = b.detach().cpu().numpy() if hasattr(b, "detach") else np.asarray(b)
        self.zero_dose_sino = b != 0

    def calcAbsorptionMask(self, target_geo):
        """Radial absorption mask exp(-a (R - r)), zero outside the grid circle
        (geometry.py:161-193).  Requires container_radius and projector_pixel_size."""
        if self.container_radius is None or self.projector_pixel_size is None:
            raise Exception(
                "container_radius and projector_pixel_size must be specified in ProjectorGeometry if "
                "absoption_coeff is used to calculate an absorption mask.")
        x = target_geo.array
        r = x.shape[0] / 2 * self.projector_pixel_size
        R = self.container_radius
        if R < r:
            raise Exception(
                "container radius is smaller than the simulation radius. container radius must be larger "
                "than simulation radius for valid reconstruction.")
        cy, cx = np.meshgrid(np.linspace(-r, r, x.shape[0]), np.linspace(-r, r, x.shape[1]))
        depth = R - np.sqrt(cx ** 2 + cy ** 2)
        coeff = 0.0 if self.absorption_coeff is None else self.absorption_coeff
        mask = np.exp(-coeff * depth)
        mask[depth < R - r] = 0
        if x.ndim == 3:
            mask = np.broadcast_to(mask[..., np.newaxis], x.shape)
        self.absorption_mask = mask


class Volume:
    """Base class of target / sinogram / reconstruction arrays (geometry.py:196-431)."""

    def __init__(self, array, proj_geo=None, **kwargs):
        self.array = array
        self.proj_geo = proj_geo
        self.file_extension = kwargs.get("file_extension")
        self.vol_type = kwargs.get("vol_type")
        self.spatial_sampling_rate = kwargs.get("spatial_sampling_rate")
        self.n_dim = np.ndim(self.array)
        shape = np.shape(self.array)
        if self.vol_type in ("recon", "target"):
            if self.n_dim == 2:
                self.nY, self.nX = shape
                self.nZ = 0
                self.resolution = None
            elif self.n_dim == 3:
                self.nY, self.nX, self.nZ = shape
                self.resolution = self.nZ
        elif self.vol_type == "sino":
            if self.n_dim == 2:
                self.nR, self.nTheta = shape
                self.nZ = 0
                self.resolution = None
            elif self.n_dim == 3:
                self.nR, self.nTheta, self.nZ = shape
                self.resolution = self.nZ

    def show(self, *args, **kwargs):
        """The reference draws the volume with matplotlib / vedo (geometry.py show()); this package has no
        display: it logs that nothing is drawn and returns, so a script that shows its results still runs
        to the end headless (the data is ``self.array``)."""
        import logging

        logging.getLogger(__name__).warning("%s.show(): no display in this package; the data is .array",
                                            type(self).__name__)

    def segmentZ(self, slices):
        if isinstance(slices, int) or (isinstance(slices, list) and len(slices) == 1):
            self.array = self.array[:, :, slices]
            self.n_dim = 2
            self.nZ = 0
            self.resolution = None
        if isinstance(slices, list):
            self.array = self.array[:, :, slices[0]:slices[1]]
            self.nZ = slices[1] - slices[0] + 1
            self.resolution = self.nZ

    def save(self, name):
        import dill

        if self.file_extension:
            name = name + self.file_extension
        with open(name, "wb") as fh:
            dill.dump(self, fh)

    def _sampling_rate(self, rate):
        if rate is not None:
            self.spatial_sampling_rate = rate
        if self.spatial_sampling_rate is None:
            self.spatial_sampling_rate = 500  # 20 micron voxels
        return self.spatial_sampling_rate

    def constructCoordVec(self, spatial_sampling_rate=None, device=None):
        """Physical coordinate vectors [xv, yv, zv] centred on 0 (geometry.py:365-430)."""
        if self.vol_type == "sino":
            return None
        rate = self._sampling_rate(spatial_sampling_rate)
        xv = np.linspace(-(self.nX - 1) / (2 * rate), (self.nX - 1) / (2 * rate), self.nX)
        yv = np.linspace(-(self.nY - 1) / (2 * rate), (self.nY - 1) / (2 * rate), self.nY)
        if self.n_dim == 2:
            zv = np.atleast_1d(0.0)
        else:
            zv = np.linspace(-(self.nZ - 1) / (2 * rate), (self.nZ - 1) / (2 * rate), self.nZ)
        self.coord_vec_list = [xv, yv, zv]
        return self.coord_vec_list

    def constructCoordGrid(self, spatial_sampling_rate=None, device=None):
        if self.vol_type == "sino":
            return None
        cv = self.constructCoordVec(spatial_sampling_rate)
        self.coord_grid_list = list(np.meshgrid(cv[0], cv[1], cv[2], indexing="ij"))
        return self.coord_grid_list


class TargetGeometry(Volume):
    """Target array (geometry.py:433-613).  2-D inputs become (nY, nX, 1)."""

    def __init__(self, target=None, stlfilename=None, resolution=None, imagefilename=None, pixels=None,
                 rot_angles=(0, 0, 0), bodies="all", binarize_image=True, clip_to_circle=True, options=None):
        self.insert = None
        self.zero_dose = None
        if target is not None:
            array = np.atleast_3d(target)
        elif imagefilename is not None and stlfilename is None:
            from PIL import Image, ImageOps

            image = Image.open(imagefilename).convert("L")
            if image.size[0] != image.size[1]:
                sq = max(image.size)
                dw, dh = sq - image.size[0], sq - image.size[1]
                image = ImageOps.expand(image, (dw // 2, dh // 2, dw - dw // 2, dh - dh // 2))
            if pixels is not None:
                image = image.resize(size=(pixels, pixels))
            image = np.array(image).astype(np.float32)
            image = image / np.max(image)
            array = np.where(image >= 0.5, 1.0, 0.0) if binarize_image else image
            array = np.atleast_3d(array)
        elif stlfilename is not None:
            raise NotImplementedError(
                "STL voxelisation uses an OpenGL slicer in the reference (vamtoolbox/voxelize.py); "
                "pass a voxel array as `target` instead")
        else:
            raise ValueError("TargetGeometry needs target= or imagefilename=")
        self.gel_inds, self.void_inds = getInds(array)
        if clip_to_circle:
            array = _data.clipToCircle(array)
        super().__init__(array=array, options=options, file_extension=".target", vol_type="target")

    def segmentZ(self, slices):
        if isinstance(slices, int) or (isinstance(slices, list) and len(slices) == 1):
            self.array = self.array[:, :, slices]
            if self.insert is not None:
                self.insert = self.insert[:, :, slices]
            self.n_dim = 2
            self.nZ = 0
            self.resolution = None
        if isinstance(slices, list):
            self.array = self.array[:, :, slices[0]:slices[1]]
            if self.insert is not None:
                self.insert = self.insert[:, :, slices[0]:slices[1]]
            self.nZ = slices[1] - slices[0] + 1
            self.resolution = self.nZ


class Sinogram(Volume):
    def __init__(self, sinogram, proj_geo, options=None):
        super().__init__(array=sinogram, proj_geo=proj_geo, options=options, file_extension=".sino",
                         vol_type="sino")


class Reconstruction(Volume):
    def __init__(self, reconstruction, proj_geo, options=None):
        super().__init__(array=reconstruction, proj_geo=proj_geo, options=options, file_extension=".recon",
                         vol_type="recon")


def loadVolume(file_name):
    import dill

    with open(file_name, "rb") as fh:
        return dill.loads(fh.read())


def getCircleMask(target):
    """Inscribed-circle mask, centre (N-1)/2 (geometry.py:682-711)."""
    if np.ndim(target) == 2:
        cy, cx = np.meshgrid(np.linspace(-1, 1, target.shape[0]), np.linspace(-1, 1, target.shape[1]))
    else:
        cy, cx, _ = np.meshgrid(np.linspace(-1, 1, target.shape[0]), np.linspace(-1, 1, target.shape[1]),
                                np.linspace(-1, 1, target.shape[2]))
    return np.array(cx ** 2 + cy ** 2 <= 1, dtype=bool)


def getInds(target):
    """Boolean gel / void masks inside the circle (geometry.py:714-733)."""
    circle = getCircleMask(target)
    return np.logical_and(target > 0, circle), np.logical_and(target == 0, circle)


def fan_beam_tables(angles, vial_width, N_screen, n_write, throw_ratio):
    """Sampling tables of rebinFanBeam (vamtoolbox/geometry.py:736-944), in float64.

    Follows the reference's formulas step by step: projector coordinate xp,
    refraction of the ray from projector pixel xp at the air/vial wall
    (xps, theta10, thetai, thetat, thetav), Fresnel transmission T (s and p
    averaged), the vial coordinate xv it samples and the differential-area
    factor np.gradient(xv) (negative values zeroed), and the sampled angle
    angle + thetav in degrees wrapped by the reference's rules (:900-909).
    Returns (xp, xv, theta_samp [nP][nA], dxv_dxp [nP], T [nP]).
    """
    angles = np.asarray(angles)
    n_angles = angles.size
    N_U = N_screen[0]
    n1, n2 = 1, n_write
    vial_width = int(vial_width)
    trp = throw_ratio * N_U
    Rv = (vial_width / 2) * np.sqrt(1 + ((vial_width) / (2 * trp)) ** 2)
    xp = np.linspace(-vial_width / 2, vial_width / 2, vial_width)
    phi = np.arctan(xp / trp)
    xps = (xp - xp * np.sqrt(1 - (1 + (xp / trp) ** 2) * (1 - (Rv / trp) ** 2))) / (1 + (xp / trp) ** 2)
    theta10 = np.arcsin(xps / Rv)
    thetai = np.arcsin(xps / Rv) + phi
    thetat = np.arcsin((n1 / n2) * np.sin(thetai))
    thetav = theta10 - thetat
    thetavD = (180 / np.pi) * thetav
    Ts = 1 - ((n1 * np.cos(thetai) - n2 * np.cos(thetat)) / ((n1 * np.cos(thetai) + n2 * np.cos(thetat)))) ** 2
    Tp = 1 - ((n1 * np.cos(thetat) - n2 * np.cos(thetai)) / ((n1 * np.cos(thetat) + n2 * np.cos(thetai)))) ** 2
    T = (Ts + Tp) / 2
    T[T < 0] = 0
    xv = (xps * np.cos(thetav)) - (np.sin(thetav) * np.sqrt((Rv ** 2) - (xps ** 2)))
    dxv_dxp = np.gradient(xv)
    dxv_dxp[T < 0] = 0
    dxv_dxp[dxv_dxp < 0] = 0
    theta_samp, _ = np.meshgrid(angles, xv)
    theta_samp = theta_samp + np.transpose(np.tile(thetavD, (n_angles, 1)))
    min_theta, max_theta = angles[0], angles[-1]
    diff_theta = abs(angles[1] - angles[0])
    theta_samp[theta_samp > max_theta] = theta_samp[theta_samp > max_theta] - 360
    theta_samp[theta_samp < min_theta] = 360 + theta_samp[theta_samp < min_theta]
    theta_samp[theta_samp > max_theta - diff_theta] = min_theta
    theta_samp[(theta_samp <= max_theta - diff_theta) & (theta_samp > max_theta)] = max_theta
    return xp, xv, theta_samp, dxv_dxp, T


def grid_search(grid, x):
    """Lower cell index and fractional position of x on an ascending grid, as
    scipy's RegularGridInterpolator (method 'linear') finds them: i =
    searchsorted(grid, x) - 1 clipped to [0, n-2], y = (x - grid[i]) /
    (grid[i+1] - grid[i]); out-of-bounds points (x < grid[0] or x > grid[-1])
    get i = -1 (interpn's fill_value=0)."""
    grid = np.asarray(grid, dtype=np.float64)
    x = np.asarray(x, dtype=np.float64)
    i = np.clip(np.searchsorted(grid, x, side="left") - 1, 0, grid.size - 2)
    y = (x - grid[i]) / (grid[i + 1] - grid[i])
    oob = (x < grid[0]) | (x > grid[-1])
    return np.where(oob, -1, i).astype(np.int32), y


_FAN_TABLES = {}


def _fan_beam_device_tables(angles, vial_width, N_screen, n_write, throw_ratio, dev):
    """Device copies of the rebinning tables, built once per geometry and device
    (a projector setup converts many sinograms with the same tables)."""
    import torch

    key = (np.asarray(angles, dtype=np.float64).tobytes(), int(vial_width), tuple(int(v) for v in N_screen),
           float(n_write), float(throw_ratio), str(dev))
    hit = _FAN_TABLES.get(key)
    if hit is not None:
        return hit
    xp, xv, theta_samp, dxv_dxp, T = fan_beam_tables(angles, vial_width, N_screen, n_write, throw_ratio)
    xi, y0 = grid_search(xp, xv)
    ti, y1 = grid_search(angles, theta_samp)
    with np.errstate(divide="ignore"):
        xw = np.stack([y0, 1 - y0, dxv_dxp, 1 / T], axis=1)
    tw = np.stack([y1, 1 - y1], axis=2)
    tabs = tuple(torch.from_numpy(np.ascontiguousarray(t)).to(dev) for t in (xi, xw, ti, tw))
    if len(_FAN_TABLES) >= 16:
        _FAN_TABLES.pop(next(iter(_FAN_TABLES)))
    _FAN_TABLES[key] = tabs
    return tabs


def rebinFanBeam(sinogram, vial_width, N_screen, n_write, throw_ratio):
    """Rebin a parallel-beam sinogram for a non-telecentric projector and a
    vial that is not index matched (vamtoolbox/geometry.py:736-944; Orth et
    al., Opt. Express 29, 11037 (2021)).

    Each output sample (xp, angle, z) is scipy interpn's bilinear sample of
    the sinogram at (xv(xp), angle + thetav(xp)), times dxv_dxp, divided by
    the Fresnel transmission T.  Like the reference, the input sinogram's
    array is replaced by its copy padded to vial_width rows, and the result
    has that shape and the input's dtype.  The per-sample work runs on the
    GPU; a numpy array comes back as numpy, a torch tensor stays on its device.
    """
    import torch

    angles = np.asarray(sinogram.proj_geo.angles)
    arr = sinogram.array
    is_torch = isinstance(arr, torch.Tensor)
    n_r, n_a, n_z = (int(d) for d in arr.shape)
    vial_width = int(vial_width)
    if n_a < 2:
        raise ValueError(f"There are {n_a} point(s) in dimension 1, but method linear requires at least 2 points.")
    if not np.all(np.diff(angles) > 0):
        raise ValueError("The points in dimension 1 must be strictly ascending")
    pd = int((vial_width - n_r) / 2)
    if is_torch:
        rows = n_r + 2 * max(pd, 0)
        rows += 1 if rows < vial_width else 0
        padded = arr
        if rows != n_r:
            padded = torch.zeros((rows, n_a, n_z), dtype=arr.dtype, device=arr.device)
            padded[max(pd, 0):max(pd, 0) + n_r] = arr
        sinogram.array = padded
    else:
        padded = arr
        if pd > 0:
            padded = np.pad(padded, ((pd, pd), (0, 0), (0, 0)), mode="constant")
        if np.shape(padded)[0] < vial_width:
            padded = np.pad(padded, ((0, 1), (0, 0), (0, 0)), mode="constant")
        sinogram.array = padded
    n_p = int(padded.shape[0])
    if n_p != vial_width:
        raise ValueError(f"There are {vial_width} points and {n_p} values in dimension 0")

    dt = arr.dtype
    if is_torch:
        dev = arr.device if arr.is_cuda else torch.device("cuda", torch.cuda.current_device())
        np_dt = np.float64 if dt == torch.float64 else (np.float32 if dt == torch.float32 else None)
        src = arr.to(dev).contiguous()
    else:
        np_dt = dt.type if dt in (np.float32, np.float64) else None
        dev = torch.device("cuda", torch.cuda.current_device())
        src = torch.from_numpy(np.ascontiguousarray(arr)).to(dev) if np_dt is not None else None
    if np_dt is None:
        raise TypeError(f"sinogram dtype {dt} is not supported (float32 or float64)")
    from . import _lib

    code = _lib.DTYPE_F64 if np_dt == np.float64 else _lib.DTYPE_F32
    with torch.cuda.device(dev):
        t_xi, t_xw, t_ti, t_tw = _fan_beam_device_tables(angles, vial_width, N_screen, n_write, throw_ratio, dev)
        out = torch.empty((n_p, n_a, n_z), dtype=src.dtype, device=dev)
        _lib.call("vam_rebin_fan", _lib.ptr(src), code, n_r, n_a, n_z, n_p, max(pd, 0), _lib.ptr(t_xi),
                  _lib.ptr(t_xw), _lib.ptr(t_ti), _lib.ptr(t_tw), _lib.ptr(out), _lib.stream_ptr())
    result = out if is_torch else out.cpu().numpy()
    return Sinogram(result, sinogram.proj_geo)
