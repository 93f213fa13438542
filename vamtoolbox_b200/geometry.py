"""Geometry data model: the reference's ``vamtoolbox.geometry`` interface.

Mirrors vamtoolbox/geometry.py (ProjectionGeometry :30-193, Volume / TargetGeometry
/ Sinogram / Reconstruction :196-659, loadVolume :662-679, getCircleMask /
getInds :682-733) so that user code written for the reference constructs the
same objects.  Arrays stay numpy on this side; the projectors move them to
the device.  ``rebinFanBeam`` (geometry.py:736-944) is not part of the
projection hot path and is not provided.
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
