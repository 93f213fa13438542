"""Curved-ray propagator on the B200: drop-in for PyTorchRayTracingPropagator.

Keeps the reference's interface (vamtoolbox/projector/pyTorchRayTrace.py:15-209):
``forward(f)`` integrates a real-space field along every ray (R6),
``backward(g)`` deposits ray energies into the grid (R5), ``inverseBackward``
builds the filtered initial sinogram used by BCLP.  The stepping, deposit and
exit logic run inside one sm_100a kernel per call (vamtoolbox_b200/csrc/raytrace.cu)
instead of ~20 ATen launches per step plus a host sync every 10 steps.

Ray starting states are built exactly like RayState.setupRaysParallel
(pyTorchRayTrace.py:1515-1666): float32 torch arithmetic on the host, then
copied to the device once.  The step size is half a voxel and the step cap
3 * N (:44-49), as in the reference.
"""
from __future__ import annotations

import ctypes
import logging

import numpy as np
import torch

from .. import _lib
from ..util.data import filterSinogram


def setup_rays_parallel(coord_vec, angles_deg, inclination_deg=0.0, ray_density=1.0):
    """x0, v0 ([num_rays, 3] float32, CPU), sinogram shape and per-ray energy.

    Restates RayState.setupRays / setupRaysParallel / resetRaysIterateToInitial
    (pyTorchRayTrace.py:1473-1700) with the same float32 torch operations, so
    the starting states are bit-identical to the reference's on the CPU.
    """
    xv, yv, zv = (np.asarray(c) for c in coord_vec)
    az = np.asarray(angles_deg) * np.pi / 180.0
    incl_deg = 0 if inclination_deg is None else inclination_deg
    incl = incl_deg * np.pi / 180.0
    dens = 1 if ray_density is None else ray_density
    nX, nY, nZ = xv.size, yv.size, zv.size
    if nZ == 1:
        shape = (round(max(nX, nY) * dens), az.size, nZ)
    else:
        shape = (round(max(nX, nY) * dens), az.size, max(round(nZ * dens), 1))
    n0min = min(np.amin(xv), np.amin(yv))
    n0max = max(np.amax(xv), np.amax(yv))
    sino_n0 = np.linspace(n0min, n0max, shape[0])
    sino_n2 = np.linspace(np.amin(zv), np.amax(zv), shape[2])
    offset = np.sqrt(n0max ** 2 + np.amax(zv) ** 2)
    f32 = lambda a: torch.as_tensor(a, dtype=torch.float32)
    inc = f32(incl)
    G0, G1, G2 = torch.meshgrid(f32(sino_n0), f32(az), f32(sino_n2), indexing="ij")
    G0, G1, G2 = torch.ravel(G0), torch.ravel(G1), torch.ravel(G2)
    nr = shape[0] * shape[1] * shape[2]
    x0 = torch.empty((nr, 3), dtype=torch.float32)
    x0[:, 0] = offset * torch.cos(G1) * torch.cos(inc)
    x0[:, 1] = offset * torch.sin(G1) * torch.cos(inc)
    x0[:, 2] = offset * torch.sin(inc)
    x0[:, 0] += -G0 * torch.sin(G1) - G2 * torch.cos(G1) * torch.sin(inc)
    x0[:, 1] += G0 * torch.cos(G1) - G2 * torch.sin(G1) * torch.sin(inc)
    x0[:, 2] += G2 * torch.cos(inc)
    v0 = torch.empty((nr, 3), dtype=torch.float32)
    v0[:, 0] = -torch.cos(G1) * torch.cos(inc)
    v0[:, 1] = -torch.sin(G1) * torch.cos(inc)
    v0[:, 2] = -torch.sin(inc)
    energy0 = float(np.float32(dens ** (-1) if sino_n2.size == 1 else dens ** (-2)))
    return x0, v0, shape, energy0


class RayPlan:
    """Owns a vam_ray_plan bound to one medium."""

    def __init__(self, coord_vec, angles_deg, index_model, attenuation_model, absorption_model, *,
                 parametrization="physical_path_length", ode_solver="forward_symplectic_euler",
                 inclination_deg=0.0, ray_density=1.0, max_num_step=None, step_size=None,
                 num_step_per_exit_check=10, device=None):
        if ode_solver is None or ode_solver not in _lib.SOLVER:
            if ode_solver == "rk4":
                raise NotImplementedError("rk4 is a placeholder in the reference (pyTorchRayTrace.py:289-292)")
            raise Exception(f"ode_solver = {ode_solver} and is not one of the available options.")
        if parametrization not in _lib.PARAM:
            raise Exception(f"eikonal_parametrization = {parametrization} and is not one of the available options.")
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        if self.device.type != "cuda":
            raise RuntimeError("the ray tracer runs on CUDA devices only")
        self.coord_vec = [np.asarray(c, dtype=np.float64) for c in coord_vec]
        xv, yv, zv = self.coord_vec
        self.grid_shape = (xv.size, yv.size, zv.size)
        x0, v0, self.sino_shape, self.energy0 = setup_rays_parallel(coord_vec, angles_deg, inclination_deg, ray_density)
        self.num_rays = x0.shape[0]
        twod = zv.size == 1
        voxel = [xv[1] - xv[0], yv[1] - yv[0], np.inf if twod else zv[1] - zv[0]]
        if step_size is None:
            step_size = voxel[0] / 2
        if max_num_step is None:
            max_num_step = int(xv.size * (2 * 1.5))
        self.step_size = float(step_size)
        self.max_num_step = int(max_num_step)
        g = _lib.RayGeom()
        g.n_x, g.n_y, g.n_z = self.grid_shape
        for d, c in enumerate(self.coord_vec):
            g.coord_min[d] = float(np.amin(c))
            g.coord_max[d] = float(np.amax(c))
            g.voxel[d] = float(voxel[d])
        g.step_size = self.step_size
        g.max_num_step = self.max_num_step
        g.num_step_per_exit_check = int(num_step_per_exit_check)
        g.parametrization = _lib.PARAM[parametrization]
        g.ode_solver = _lib.SOLVER[ode_solver]
        g.num_rays = self.num_rays
        g.device = self.device.index
        x0d = x0.to(self.device).contiguous()
        v0d = v0.to(self.device).contiguous()
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.call("vam_ray_plan_create", ctypes.byref(g), _lib.ptr(x0d), _lib.ptr(v0d), self.energy0, ctypes.byref(h))
        self._h = h
        self.x0, self.v0 = x0, v0
        self.bind_medium(index_model, attenuation_model, absorption_model)

    def bind_medium(self, index_model, attenuation_model, absorption_model):
        m = _lib.RayMedium()
        keep = []
        nk, nsur, lR, lp, ng, gg = index_model.kernel_fields()
        m.index_kind, m.n_sur, m.lune_R, m.lune_p = nk, nsur, lR, lp
        if ng is not None:
            ng, gg = ng.to(self.device), gg.to(self.device)
            keep += [ng, gg]
            m.n_grid_dev, m.grad_n_grid_dev = ng.data_ptr(), gg.data_ptr()
        if attenuation_model is None:
            m.atten_kind = _lib.ALPHA_ZERO
        else:
            ak, av, aR, ag = attenuation_model.kernel_fields()
            m.atten_kind, m.atten_value, m.atten_R = ak, av, aR
            if ag is not None:
                ag = ag.to(self.device)
                keep.append(ag)
                m.atten_grid_dev = ag.data_ptr()
        if absorption_model is None:
            raise ValueError("the ray tracer needs an absorption model (alpha at the grid points)")
        ab = absorption_model.alpha_at_grid().to(self.device).contiguous()
        keep.append(ab)
        m.absorb_at_grid_dev = ab.data_ptr()
        self.absorb_at_grid = ab
        with torch.cuda.device(self.device):
            _lib.call("vam_ray_set_medium", self._h, ctypes.byref(m), _lib.stream_ptr(torch.cuda.current_stream(self.device)))
            torch.cuda.current_stream(self.device).synchronize()
        self._medium_keep = keep
        self.has_trajectories = False  # a new medium makes the cached paths stale
        self.cached_rays = 0

    def trajectory_bytes(self, rays=None):
        """Device bytes of the trajectory cache of ``rays`` rays (default: every ray): 16 per ray and step
        of the cap, 4 per ray."""
        rays = self.num_rays if rays is None else int(rays)
        return (16 * max(self.max_num_step, 1) + 4) * rays

    def _cacheable_rays(self, limit_bytes):
        """The rays vam_ray_prepare_trajectories caches under limit_bytes: every ray when they fit, else the
        largest multiple of 32 (rays 0 .. m - 1; the rest are traced every call)."""
        m = min(self.num_rays, int(limit_bytes) // (16 * max(self.max_num_step, 1) + 4))
        return m if m == self.num_rays else m - m % 32

    def prepare_trajectories(self, limit_bytes=None):
        """Trace the rays once and keep every step's position and attenuance (vam_ray_prepare_trajectories),
        so later integrate / deposit calls stream them instead of re-tracing (bit-identical results).  The
        paths depend on the medium only.  ``limit_bytes`` defaults to half of the device's free memory;
        when not every ray fits, the first ``cached_rays`` rays (a multiple of 32) are cached and the rest
        traced every call.  Allocates: not during a graph capture.  False when the configuration has no
        cached path (it serves 3-D grid media, physical path length, symplectic Euler) or not even 32 rays
        fit the limit or the device; the plan then keeps tracing."""
        if limit_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            limit_bytes = free // 2
        self.cached_rays = 0
        try:
            with torch.cuda.device(self.device):
                _lib.call("vam_ray_prepare_trajectories", self._h, int(limit_bytes), self._s())
                torch.cuda.current_stream(self.device).synchronize()
        except _lib.VamError as exc:
            if exc.code in (_lib.VAM_ERR_NOTSUP, _lib.VAM_ERR_NOMEM):
                self.has_trajectories = False
                return False
            raise
        self.has_trajectories = True
        self.cached_rays = self._cacheable_rays(limit_bytes)
        return True

    def drop_trajectories(self):
        """Free the trajectory cache (later calls trace again)."""
        with torch.cuda.device(self.device):
            _lib.call("vam_ray_drop_trajectories", self._h)
        self.has_trajectories = False
        self.cached_rays = 0

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.load().vam_ray_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _s(self):
        return _lib.stream_ptr(torch.cuda.current_stream(self.device))

    def integrate(self, f, out=None):
        f = f.to(device=self.device, dtype=torch.float32).reshape(self.grid_shape).contiguous()
        if out is None:
            out = torch.empty(self.num_rays, dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.call("vam_ray_integrate", self._h, _lib.ptr(f), _lib.ptr(out), self._s())
        return out

    def deposit(self, g, out=None):
        g = g.to(device=self.device, dtype=torch.float32).reshape(-1).contiguous()
        if g.numel() != self.num_rays:
            raise ValueError(f"expected {self.num_rays} ray energies, got {g.numel()}")
        if out is None:
            out = torch.empty(self.grid_shape, dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.call("vam_ray_deposit", self._h, _lib.ptr(g), _lib.ptr(out), self._s())
        return out

    def grad_alpha(self, f, w, grad_att=None, grad_abs=None):
        f = f.to(device=self.device, dtype=torch.float32).reshape(self.grid_shape).contiguous()
        w = w.to(device=self.device, dtype=torch.float32).reshape(-1).contiguous()
        with torch.cuda.device(self.device):
            _lib.call("vam_ray_grad_alpha", self._h, _lib.ptr(f), _lib.ptr(w), _lib.ptr(grad_att), _lib.ptr(grad_abs),
                      self._s())

    def record(self):
        """The integrate operator as a CSR matrix (one row per ray, C-order voxel columns): returns
        (row_ptr int64 [num_rays + 1], cols int32, vals float32) on the device, uncoalesced (a voxel met
        twice appears twice, as in the reference before it coalesces)."""
        nr = self.num_rays
        cnt = torch.empty(nr, dtype=torch.int64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.call("vam_ray_record_count", self._h, _lib.ptr(cnt), self._s())
            row_ptr = torch.zeros(nr + 1, dtype=torch.int64, device=self.device)
            torch.cumsum(cnt, 0, out=row_ptr[1:])
            nnz = int(row_ptr[-1].item())
            cols = torch.empty(max(nnz, 1), dtype=torch.int32, device=self.device)
            vals = torch.empty(max(nnz, 1), dtype=torch.float32, device=self.device)
            _lib.call("vam_ray_record_fill", self._h, _lib.ptr(row_ptr), _lib.ptr(cols), _lib.ptr(vals), self._s())
        return row_ptr, cols[:nnz], vals[:nnz]

    def active_at_cap(self):
        v = ctypes.c_int64()
        with torch.cuda.device(self.device):
            _lib.call("vam_ray_active_at_cap", self._h, ctypes.byref(v))
        return int(v.value)


class PyTorchRayTracingPropagator:
    """B200 ray-tracing propagator (pyTorchRayTrace.py:15-209)."""

    def __init__(self, target_geo, proj_geo, output_torch_tensor=False, device=None):
        self.logger = logging.getLogger(__name__)
        self.target_geo = target_geo
        self.proj_geo = proj_geo
        self.output_torch_tensor = output_torch_tensor
        if proj_geo.ray_trace_ray_config not in (None, "parallel"):
            raise Exception(f"Ray config: {proj_geo.ray_trace_ray_config} is not one of the supported string: 'parallel', 'cone'.")
        if proj_geo.ray_trace_method not in (None, "eikonal", "hybrid", "snells"):
            raise Exception(f"ray_trace_method = {proj_geo.ray_trace_method} is not supported")
        coord_vec = target_geo.constructCoordVec()
        im = proj_geo.index_model
        self.tracing_step_size = float(im.voxel_size[0].cpu().numpy() / 2)
        self.max_num_step = int(target_geo.array.shape[0] * (2 * 1.5))
        self.plan = RayPlan(coord_vec, proj_geo.angles, im, proj_geo.attenuation_model, proj_geo.absorption_model,
                            parametrization=proj_geo.eikonal_parametrization or "physical_path_length",
                            ode_solver=proj_geo.ray_trace_ode_solver,
                            inclination_deg=proj_geo.inclination_angle or 0.0,
                            ray_density=proj_geo.ray_density if proj_geo.ray_density is not None else 1.0,
                            max_num_step=self.max_num_step, step_size=self.tracing_step_size, device=device)
        self.device = self.plan.device
        self.sino_shape = self.plan.sino_shape

    def _report_cap(self):
        if self.logger.isEnabledFor(logging.ERROR):
            n = self.plan.active_at_cap()
            if n:
                self.logger.error(f"Some rays are still active when max_num_step ({self.max_num_step}) is reached. "
                                  f"Rays active: {n}/{self.plan.num_rays}.")

    def forward_t(self, f, out=None):
        if not isinstance(f, torch.Tensor):
            f = torch.as_tensor(np.asarray(f), device=self.device)
        return self.plan.integrate(f, out)

    def backward_t(self, g, out=None):
        if not isinstance(g, torch.Tensor):
            g = torch.as_tensor(np.asarray(g), device=self.device)
        return self.plan.deposit(g, out)

    def forward(self, f):
        g = self.forward_t(f)
        if self.output_torch_tensor:
            return g
        return g.cpu().numpy()

    def backward(self, ray_energy_0):
        d = self.backward_t(ray_energy_0)
        if self.output_torch_tensor:
            return d
        return np.squeeze(d.cpu().numpy())

    def buildPropagationMatrix(self):
        """The forward propagation matrix (pyTorchRayTrace.py:169-197): rows = rays, columns = voxels
        (C order over the [nX][nY][nZ] grid), coalesced; a torch sparse COO tensor when
        ``output_torch_tensor``, else a scipy.sparse.coo_array."""
        row_ptr, cols, vals = self.plan.record()
        nvox = int(np.prod(self.plan.grid_shape))
        rows = torch.repeat_interleave(torch.arange(self.plan.num_rays, device=self.device),
                                       row_ptr[1:] - row_ptr[:-1])
        A = torch.sparse_coo_tensor(torch.vstack((rows, cols.to(torch.int64))), vals,
                                    size=(self.plan.num_rays, nvox), device=self.device,
                                    check_invariants=False).coalesce()  # indices in range by construction
        if self.output_torch_tensor:
            return A
        import scipy.sparse

        idx = A.indices().cpu().numpy()
        return scipy.sparse.coo_array((A.values().cpu().numpy(), (idx[0], idx[1])), shape=tuple(A.shape))

    def inverseBackward(self, f, filter_option="ram-lak", **kwargs):
        """Filtered initial sinogram (pyTorchRayTrace.py:135-166)."""
        f = torch.as_tensor(np.asarray(f) if not isinstance(f, torch.Tensor) else f, device=self.device,
                            dtype=torch.float64).reshape(self.plan.grid_shape)
        a = self.plan.absorb_at_grid.to(torch.float64)
        f = f / a ** 2.0
        f[torch.isnan(f) | torch.isinf(f)] = 0.0
        g0 = self.forward_t(f.to(torch.float32)).reshape(self.sino_shape).double().cpu().numpy()
        g0 = filterSinogram(g0, filter_option).ravel()
        g0 *= np.pi / (2 * self.proj_geo.n_angles)
        if self.output_torch_tensor:
            return torch.as_tensor(g0, device=self.device)
        return g0

    # placeholders of the reference's interface with no body there either (pyTorchRayTrace.py:199-209)
    def perAngleTrace(self):
        pass

    def perZTrace(self):
        pass

    def perRayTrace(self):
        pass
