"""Generate the golden vectors under tests/golden/ by running the reference.

Run in a checkout that has the reference tree (default /root/reference, or
VAM_REFERENCE_ROOT):

    python tests/golden/make_golden.py

Every array stored here is produced by the reference's own Python code
(Projector3DParallelPython, Projector2DParallelPython, the PyTorch ray tracer
on the CPU, the CAL / OSMO / BCLP optimizers, ImageSeq and rebinFanBeam),
loaded through
oracle/refload.py.  The only restated routine on that path is
skimage.transform.warp (absent here), see oracle/refload.py.  Inputs are
seeded synthetic targets; sizes are small so the fixtures stay a few hundred KB.
"""
from __future__ import annotations

import sys
import warnings
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import refload  # noqa: E402

OUT = Path(__file__).resolve().parent


def ellipses_target(n, nz, rng, n_ell=4):
    y, x = np.mgrid[:n, :n] - (n - 1) / 2
    t = np.zeros((n, n, nz))
    for z in range(nz):
        img = np.zeros((n, n))
        for _ in range(n_ell):
            cy, cx = rng.uniform(-n / 4, n / 4, 2)
            a, b = rng.uniform(n / 10, n / 3, 2)
            th = rng.uniform(0, np.pi)
            xr = (x - cx) * np.cos(th) + (y - cy) * np.sin(th)
            yr = -(x - cx) * np.sin(th) + (y - cy) * np.cos(th)
            img[(xr / a) ** 2 + (yr / b) ** 2 <= 1] = 1.0
        t[:, :, z] = img
    return t


def parallel_cases(vam):
    geo = vam.geometry
    P3 = vam.projector.Projector3DParallel.Projector3DParallelPython
    out = {}
    rng = np.random.default_rng(1234)
    for tag, n, nz, na, full in (("even", 24, 3, 16, 360.0), ("odd", 25, 2, 13, 180.0)):
        x = rng.uniform(0, 1, (n, n, nz))
        ang = np.linspace(0, full, na, endpoint=False)
        tg = geo.TargetGeometry(target=x.copy(), clip_to_circle=False)
        pg = geo.ProjectionGeometry(ang, "parallel", CUDA=False, attenuation_field=np.zeros((n, n, nz)))
        A = P3(tg, pg)
        b = A.forward(x.copy())
        bb = rng.uniform(0, 1, b.shape)
        xb = A.backward(bb.copy())
        out[f"{tag}_x"] = x
        out[f"{tag}_angles"] = ang
        out[f"{tag}_fwd"] = b
        out[f"{tag}_b"] = bb
        out[f"{tag}_bwd"] = xb
    # occlusion: an opaque insert (attenuation_field > 0)
    n, nz, na = 24, 2, 12
    x = ellipses_target(n, nz, rng)
    ins = np.zeros((n, n, nz))
    ins[9:13, 14:18, :] = 1.0
    ins[4:6, 6:9, 1] = 1.0
    ang = np.linspace(0, 360, na, endpoint=False)
    tg = geo.TargetGeometry(target=x.copy(), clip_to_circle=False)
    pg = geo.ProjectionGeometry(ang, "parallel", CUDA=False, attenuation_field=ins.copy())
    A = P3(tg, pg)
    b = A.forward(x.copy())
    bb = rng.uniform(0, 1, b.shape)
    out["occ_x"] = x
    out["occ_insert"] = ins
    out["occ_angles"] = ang
    out["occ_sino"] = A.occ_sinogram
    out["occ_fwd"] = b
    out["occ_b"] = bb
    out["occ_bwd"] = A.backward(bb.copy())
    # 2D class (reachable after segmentZ(int)): forward clips its input
    P2 = vam.projector.Projector2DParallel.Projector2DParallelPython
    n, na = 20, 10
    x2 = rng.uniform(0, 1, (n, n))
    ang = np.linspace(0, 360, na, endpoint=False)
    tg = geo.TargetGeometry(target=x2.copy(), clip_to_circle=False)
    tg.segmentZ(0)
    # Projector2DParallel.py:205 reads target_geo.target, which TargetGeometry
    # never sets (AttributeError in the reference); alias it to the array.
    tg.target = tg.array
    pg = geo.ProjectionGeometry(ang, "parallel", CUDA=False)
    A2 = P2(tg, pg)
    out["p2_x"] = x2
    out["p2_angles"] = ang
    out["p2_fwd"] = A2.forward(x2.copy())
    bb = rng.uniform(0, 1, (n, na))
    out["p2_b"] = bb
    out["p2_bwd"] = A2.backward(bb.copy())
    # absorption mask (geometry.py:161-193) for a 3-D target
    n = 24
    tg = geo.TargetGeometry(target=np.ones((n, n, 2)))
    pg = geo.ProjectionGeometry(np.array([0.0]), "parallel", projector_pixel_size=0.01,
                                absorption_coeff=2.0, container_radius=0.15)
    pg.calcAbsorptionMask(tg)
    out["mask"] = np.ascontiguousarray(pg.absorption_mask[:, :, 0])
    out["mask_params"] = np.array([0.01, 2.0, 0.15])
    np.savez_compressed(OUT / "parallel.npz", **out)


def ray_cases(vam):
    import torch

    geo, med = vam.geometry, vam.medium
    RT = vam.projector.pyTorchRayTrace
    out = {}
    rng = np.random.default_rng(99)
    for tag, (n, nz) in (("r3", (12, 6)), ("r2", (14, 1))):
        t = rng.uniform(0, 1, (n, n, nz))
        tg = geo.TargetGeometry(target=t if nz > 1 else t[:, :, 0])
        cv = tg.constructCoordVec()
        xg, yg, zg = np.meshgrid(*cv, indexing="ij")
        R = np.amax(cv[0])
        r2 = (xg ** 2 + yg ** 2) / R ** 2
        n_x = 1.30 + 0.05 * r2 + 0.01 * rng.uniform(-1, 1, xg.shape)
        alpha_x = 20.0 * (1 + 0.3 * rng.uniform(-1, 1, xg.shape))
        im = med.IndexModel(cv, type="interpolation", form="freeform", n_x=torch.as_tensor(n_x))
        am = med.AttenuationModel(cv, type="interpolation", form="freeform", alpha_x=torch.as_tensor(alpha_x))
        ang = np.linspace(0, 360, 5, endpoint=False)
        pg = geo.ProjectionGeometry(ang, "ray_trace", CUDA=False, index_model=im, attenuation_model=am,
                                    absorption_model=am, ray_trace_method="eikonal",
                                    eikonal_parametrization="physical_path_length",
                                    ray_trace_ode_solver="forward_symplectic_euler",
                                    ray_trace_ray_config="parallel", inclination_angle=0.0, ray_density=1)
        P = RT.PyTorchRayTracingPropagator(tg, pg)
        f = rng.uniform(0, 1, tg.array.shape)
        g = P.forward(f.copy())
        gin = rng.uniform(0, 1, g.shape).astype(np.float32)
        dose = P.backward(gin.copy())
        out[f"{tag}_xv"], out[f"{tag}_yv"], out[f"{tag}_zv"] = cv
        out[f"{tag}_n"] = n_x
        out[f"{tag}_alpha"] = alpha_x
        out[f"{tag}_angles"] = ang
        out[f"{tag}_x0"] = P.ray_state.x_0.numpy()
        out[f"{tag}_v0"] = P.ray_state.v_0.numpy()
        out[f"{tag}_f"] = f
        out[f"{tag}_fwd"] = g
        out[f"{tag}_g"] = gin
        out[f"{tag}_bwd"] = dose
        out[f"{tag}_step"] = np.array([P.tracing_step_size, P.max_num_step])
        # the propagation matrix (coalesced COO) of the same tracer
        M = P.buildPropagationMatrix()
        out[f"{tag}_mat_rows"], out[f"{tag}_mat_cols"] = M.row.astype(np.int64), M.col.astype(np.int64)
        out[f"{tag}_mat_vals"], out[f"{tag}_mat_shape"] = M.data.astype(np.float64), np.array(M.shape)
    # analytic media: homogeneous index (n_sur = 1) and absorbing cylinder
    n, nz = 12, 4
    tg = geo.TargetGeometry(target=np.ones((n, n, nz)))
    cv = tg.constructCoordVec()
    im = med.IndexModel(cv, type="analytical", form="homogeneous", n_sur=1.0)
    am = med.AttenuationModel(cv, type="analytical", form="homogeneous_cylinder", R=1, alpha_internal=30.0)
    ang = np.linspace(0, 360, 4, endpoint=False)
    pg = geo.ProjectionGeometry(ang, "ray_trace", CUDA=False, index_model=im, attenuation_model=am,
                                absorption_model=am, ray_trace_method="eikonal",
                                eikonal_parametrization="physical_path_length",
                                ray_trace_ode_solver="forward_symplectic_euler",
                                ray_trace_ray_config="parallel", inclination_angle=0.0, ray_density=1)
    P = RT.PyTorchRayTracingPropagator(tg, pg)
    f = rng.uniform(0, 1, tg.array.shape)
    out["ha_xv"], out["ha_yv"], out["ha_zv"] = cv
    out["ha_angles"] = ang
    out["ha_f"] = f
    out["ha_fwd"] = P.forward(f.copy())
    gin = rng.uniform(0, 1, out["ha_fwd"].shape).astype(np.float32)
    out["ha_g"] = gin
    out["ha_bwd"] = P.backward(gin.copy())
    out["ha_params"] = np.array([1.0, 30.0, np.amax(cv[0]) - np.amin(cv[0])])
    np.savez_compressed(OUT / "raytrace.npz", **out)


def algebraic_cases(vam):
    """The reference's PyTorchAlgebraicPropagator on the 2-D (one z layer) propagation matrix of the r2
    tracer case, z-tiled over a three-layer volume, loaded from a SciPy .npz file."""
    import os
    import tempfile

    import scipy.sparse

    R = np.load(OUT / "raytrace.npz")
    shape = tuple(R["r2_mat_shape"])
    M = scipy.sparse.coo_matrix((R["r2_mat_vals"], (R["r2_mat_rows"], R["r2_mat_cols"])), shape=shape)
    rng = np.random.default_rng(11)
    n = int(round(np.sqrt(shape[1])))
    x = rng.uniform(0, 1, (n, n, 3))
    b = rng.uniform(0, 1, shape[0] * 3)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "propagation_matrix.npz")
        scipy.sparse.save_npz(path, M.tocsr())
        tg = vam.geometry.TargetGeometry(target=x.copy())
        pg = vam.geometry.ProjectionGeometry(np.linspace(0, 360, 5, endpoint=False), "algebraic", CUDA=False,
                                             loading_path_for_matrix=path)
        A = vam.projector.pyTorchAlgebraicPropagation.PyTorchAlgebraicPropagator(tg, pg)
        fwd, bwd = A.forward(x), A.backward(b)
    np.savez_compressed(OUT / "algebraic.npz", x=x, b=b, fwd=np.asarray(fwd), bwd=np.asarray(bwd),
                        z_tiling=np.array(A.z_tiling))


def ray_autograd_cases(vam):
    """Gradients of L = <w, forward(f)> with respect to f and to the attenuation grid, taken by
    autograd through the reference's own ray tracer (inference_mode neutralised)."""
    import torch

    RT, MED = refload.load_autograd_tracer()
    geo = vam.geometry
    rng = np.random.default_rng(7)
    n, nz = 12, 6
    tg = geo.TargetGeometry(target=rng.uniform(0, 1, (n, n, nz)))
    cv = tg.constructCoordVec()
    xg, yg, _ = np.meshgrid(*cv, indexing="ij")
    R = np.amax(cv[0])
    n_x = 1.30 + 0.05 * (xg ** 2 + yg ** 2) / R ** 2
    alpha_np = 20.0 * (1 + 0.3 * rng.uniform(-1, 1, xg.shape))
    alpha_x = torch.as_tensor(alpha_np).requires_grad_(True)
    im = MED.IndexModel(cv, type="interpolation", form="freeform", n_x=torch.as_tensor(n_x))
    am = MED.AttenuationModel(cv, type="interpolation", form="freeform", alpha_x=alpha_x)
    ab = MED.AttenuationModel(cv, type="analytical", form="homogeneous_cylinder", R=1, alpha_internal=10.0)
    ang = np.linspace(0, 360, 5, endpoint=False)
    pg = geo.ProjectionGeometry(ang, "ray_trace", CUDA=False, index_model=im, attenuation_model=am,
                                absorption_model=ab, ray_trace_method="eikonal",
                                eikonal_parametrization="physical_path_length",
                                ray_trace_ode_solver="forward_symplectic_euler", ray_trace_ray_config="parallel",
                                inclination_angle=0.0, ray_density=1)
    P = RT.PyTorchRayTracingPropagator(tg, pg)
    P.output_torch_tensor = True
    f = rng.uniform(0, 1, (n, n, nz))
    f_leaf = torch.as_tensor(f).requires_grad_(True)
    g = P.forward(f_leaf * 1.0)  # the reference scales its input in place: hand it a non-leaf copy
    w = rng.uniform(0, 1, tuple(g.shape))
    L = (g * torch.as_tensor(w, dtype=g.dtype)).sum()
    L.backward()
    out = {"ag_xv": cv[0], "ag_yv": cv[1], "ag_zv": cv[2], "ag_n": n_x, "ag_alpha": alpha_np, "ag_angles": ang,
           "ag_f": f, "ag_w": w, "ag_fwd": g.detach().numpy(), "ag_L": np.array(float(L.detach())),
           "ag_grad_f": f_leaf.grad.numpy(), "ag_grad_alpha": alpha_x.grad.numpy(),
           "ag_absorption": np.array([1.0, 10.0])}
    np.savez_compressed(OUT / "ray_autograd.npz", **out)


def optimizer_cases(vam):
    geo = vam.geometry
    out = {}
    rng = np.random.default_rng(7)
    n, nz = 24, 2
    t = ellipses_target(n, nz, rng)
    ang = np.linspace(0, 360, 18, endpoint=False)
    out["target"] = t
    out["angles"] = ang

    def run(method, **kw):
        tg = geo.TargetGeometry(target=t.copy())
        pg = geo.ProjectionGeometry(ang, "parallel", CUDA=False, attenuation_field=np.zeros((n, n, nz)))
        opts = refload.fresh_options(vam, method=method, **kw)
        return vam.optimize.optimize(tg, pg, opts)

    s, r, e = run("CAL", n_iter=5, learning_rate=0.4, d_h=0.5, sigmoid=0.01)
    out["cal_sino"], out["cal_recon"], out["cal_err"] = s.array, r.array, e
    s, r, e = run("OSMO", n_iter=4, d_h=0.8, d_l=0.7, filter="ram-lak")
    out["osmo_sino"], out["osmo_recon"], out["osmo_err"] = s.array, r.array, e
    s, r, e = run("FBP", n_iter=1, filter="ram-lak")
    out["fbp_sino"], out["fbp_recon"], out["fbp_err"] = s.array, r.array, e
    # BCLP grayscale with a generalised-logistic response model
    tgray = np.clip(t * 0.8 + 0.1 * rng.uniform(0, 1, t.shape), 0, 1)
    out["bclp_target"] = tgray
    rm = vam.response.ResponseModel(B=12, M=0.6)
    tg = geo.TargetGeometry(target=tgray.copy())
    pg = geo.ProjectionGeometry(ang, "parallel", CUDA=False, attenuation_field=np.zeros((n, n, nz)))
    opts = refload.fresh_options(vam, method="BCLP", n_iter=4, p=2, q=1, eps=0.05, learning_rate=0.002,
                                 response_model=rm, filter="ram-lak")
    sino, dose, mapped, logs = vam.optimize.optimize(tg, pg, opts, output="full")
    out["bclp_sino"], out["bclp_dose"], out["bclp_mapped"] = sino.array, dose.array, mapped.array
    out["bclp_loss"] = logs.loss
    out["bclp_norms"] = np.stack([logs.l0, logs.l1, logs.l2, logs.lf, logs.l0_eps0, logs.l1_eps0,
                                  logs.l2_eps0, logs.lf_eps0])
    # BCLP with the fourth-power band norm and per-voxel weights (1 inside the target, 0.5 outside)
    w = np.where(tgray > 0.15, 1.0, 0.5)
    out["bclp4_weight"] = w
    tg = geo.TargetGeometry(target=tgray.copy())
    pg = geo.ProjectionGeometry(ang, "parallel", CUDA=False, attenuation_field=np.zeros((n, n, nz)))
    opts = refload.fresh_options(vam, method="BCLP", n_iter=4, p=4, q=1, eps=0.05, weight=w, learning_rate=0.02,
                                 response_model=rm, filter="ram-lak")
    sino, dose, mapped, logs = vam.optimize.optimize(tg, pg, opts, output="full")
    out["bclp4_sino"], out["bclp4_dose"], out["bclp4_loss"] = sino.array, dose.array, logs.loss
    # 2-D CAL: a single slice (the reference stores 2-D targets as n x n x 1 arrays)
    t2 = t[:, :, 0].copy()
    out["cal2d_target"] = t2
    tg = geo.TargetGeometry(target=t2.copy())
    pg = geo.ProjectionGeometry(ang, "parallel", CUDA=False, attenuation_field=np.zeros((n, n, 1)))
    opts = refload.fresh_options(vam, method="CAL", n_iter=5, learning_rate=0.4, d_h=0.5, sigmoid=0.01)
    s2, r2, e2 = vam.optimize.optimize(tg, pg, opts)
    out["cal2d_sino"], out["cal2d_recon"], out["cal2d_err"] = s2.array, r2.array, e2
    # response model tables
    out["resp_f"], out["resp_map"], out["resp_dmap"] = rm.interp_f_0, rm.interp_map_0, rm.interp_dmapdf_0
    out["resp_inv_probe"] = rm.map_inv(np.linspace(-0.1, 1.1, 37))
    # PM (L-BFGS-B) few iterations
    tg = geo.TargetGeometry(target=t.copy())
    pg = geo.ProjectionGeometry(ang, "parallel", CUDA=False, attenuation_field=np.zeros((n, n, nz)))
    opts = refload.fresh_options(vam, method="PM", n_iter=3, d_h=0.8, d_l=0.6, rho_1=1, rho_2=1, p=2)
    s, r, e = vam.optimize.optimize(tg, pg, opts)
    out["pm_sino"], out["pm_recon"], out["pm_err"] = s.array, r.array, e
    # filters
    for name in ("ram-lak", "shepp-logan", "cosine", "hamming", "hanning"):
        out["filt_" + name] = vam.util.data._get_fourier_filter(64, name)[:, 0]
    sino = rng.uniform(0, 1, (24, 5, 2))
    out["filt_sino_in"] = sino
    out["filt_sino_ramlak"] = vam.util.data.filterSinogram(sino.copy(), "ram-lak")
    out["filt_osmo"] = vam.util.data.filterTargetOSMO(t.copy(), "ram-lak")
    np.savez_compressed(OUT / "optim.npz", **out)


# Frame-sequence configurations: (sinogram dtype, ImageConfig keywords).  Frames are 64 x 48.
FORMAT_CASES = [
    ("float64", {}),
    ("float64", {"normalization_percentile": 99.5}),
    ("float32", {"normalization_percentile": 99.0, "intensity_scale": 0.8}),
    ("float64", {"invert_u": True, "invert_v": True, "u_offset": 3, "v_offset": -2}),
    ("float64", {"rotate_angle": 30.0, "normalization_percentile": 100}),
    ("float32", {"rotate_angle": -12.5, "invert_u": True}),
    ("float64", {"size_scale": 1.5, "normalization_percentile": 98}),
    ("float32", {"size_scale": 0.7}),
    ("float64", {"array_num": 3, "array_offset": 10, "v_offset": 1, "normalization_percentile": 99}),
    ("float64", {"array_num": 2, "array_offset": 12}),
    ("float64", {"bit_depth": 10, "normalization_percentile": 99}),
    ("float64", {"bit_depth": 16, "intensity_scale": 300.0}),
    ("float32", {"bit_depth": 32, "intensity_scale": 3e7}),
    ("float64", {"rotate_angle": 90.0, "size_scale": 1.25, "invert_v": True, "normalization_percentile": 97.5,
                 "bit_depth": 12}),
    ("float32", {"normalization_percentile": 50, "invert_v": True, "array_num": 0}),
]
# Fan-beam rebinning cases: (nR, nA, nZ, vial_width, dtype, n_write, throw_ratio).
REBIN_CASES = [
    (20, 36, 5, 25, "float64", 1.5, 1.7),
    (30, 72, 3, 30, "float64", 1.48, 2.0),
    (16, 90, 4, 21, "float32", 1.52, 1.2),
    (40, 60, 2, 47, "float64", 1.33, 3.5),
]


def format_cases(vam):
    """ImageSeq frames (vamtoolbox/imagesequence.py:85-174) and rebinFanBeam
    (vamtoolbox/geometry.py:736-944), both run by the reference itself."""
    import json

    ims = vam.imagesequence
    rng = np.random.default_rng(7)
    out = {}
    for i, (dt, kw) in enumerate(FORMAT_CASES):
        # values on a 1/1024 lattice: exact in float32 and float64, and the fixture compresses
        sino = (rng.integers(0, 3 * 1024, size=(24, 7, 20)) / 1024.0).astype(dt)
        cfg = ims.ImageConfig((64, 48), **kw)
        out[f"seq{i}_sino"] = sino
        out[f"seq{i}_cfg"] = np.array(json.dumps(kw))
        out[f"seq{i}_frames"] = np.stack(ims.ImageSeq(cfg, sino.copy()).images)
    for i, (nr, na, nz, vw, dt, n_write, throw) in enumerate(REBIN_CASES):
        angles = np.linspace(0, 360, na, endpoint=False)
        arr = (rng.integers(0, 1024, size=(nr, na, nz)) / 1024.0).astype(dt)
        pg = vam.geometry.ProjectionGeometry(angles, ray_type="parallel", CUDA=False)
        res = vam.geometry.rebinFanBeam(vam.geometry.Sinogram(arr.copy(), pg), vw, (1920, 1080), n_write, throw)
        out[f"rebin{i}_sino"] = arr
        out[f"rebin{i}_angles"] = angles
        out[f"rebin{i}_args"] = np.array([vw, 1920, 1080, n_write, throw])
        out[f"rebin{i}_out"] = res.array
    np.savez_compressed(OUT / "formats.npz", **out)


VEC_CASES = [(np.linspace(0, 360, 12, endpoint=False), 0.0), (np.linspace(0, 360, 36, endpoint=False), 15.0),
             (np.array([0.0, 33.3, 90.0, 181.0, 270.5]), -30.0), (np.linspace(0, 180, 8), 50.0)]


def vecgeom_cases(vam):
    """The reference's own genVectorsAstra rows (vamtoolbox/projector/genVectorsAstra.py:4-53): the
    inclined (laminography) geometry its CUDA projector hands to ASTRA."""
    import importlib

    gv = importlib.import_module("vamtoolbox.projector.genVectorsAstra").genVectorsAstra
    out = {}
    for i, (ang, inc) in enumerate(VEC_CASES):
        out[f"v{i}_angles"] = ang
        out[f"v{i}_incline"] = np.array(inc)
        out[f"v{i}_vectors"] = gv(ang, inc)
    out["cone_vectors"] = gv(np.array([0.0, 45.0, 100.0]), 10.0, cone_angle=5.0, distance_origin_source=250.0)
    np.savez_compressed(OUT / "vecgeom.npz", **out)


def occ2d_cases(vam):
    """Projector2DParallelPython with a digitised occlusion (Projector2DParallel.py:70-143, 145-247):
    the occlusion sinogram, forward and backward, for an even and an odd slice with occluders whose
    detector coordinates stay on the detector (np.digitize never wraps to the last bin)."""
    geo = vam.geometry
    P2 = vam.projector.Projector2DParallel.Projector2DParallelPython
    rng = np.random.default_rng(4321)
    out = {}
    for tag, n, na, boxes in (("even", 20, 12, ((8, 12, 11, 15), (5, 7, 6, 9))),
                              ("odd", 21, 9, ((9, 13, 4, 7),))):
        occ = np.zeros((n, n), dtype=bool)
        for r0, r1, c0, c1 in boxes:
            occ[r0:r1, c0:c1] = True
        x = rng.uniform(0, 1, (n, n))
        ang = np.linspace(0, 360, na, endpoint=False) + 0.7
        tg = geo.TargetGeometry(target=x.copy(), clip_to_circle=False)
        tg.segmentZ(0)
        tg.target = tg.array  # Projector2DParallel.py:205 reads target_geo.target (see parallel_cases)
        pg = geo.ProjectionGeometry(ang, "parallel", CUDA=False, occlusion=occ.copy())
        A2 = P2(tg, pg)
        b = rng.uniform(0, 1, (n, na))
        out[f"{tag}_occ"] = occ
        out[f"{tag}_x"] = x
        out[f"{tag}_angles"] = ang
        out[f"{tag}_sino"] = A2.occ_sinogram
        out[f"{tag}_fwd"] = A2.forward(x.copy())
        out[f"{tag}_b"] = b
        out[f"{tag}_bwd"] = A2.backward(b.copy())
        out[f"{tag}_bwd_noclip"] = A2.backward(b.copy(), clipping=False)
    # occluders in the corners: at some angles their detector coordinate falls below the first bin, where
    # np.digitize gives index -1 (the last bin's value); the reference then pairs its per-bin minima with
    # the bins in a shifted order ("wrap", kept), or raises when the last bin is occupied too ("clash")
    for tag, boxes in (("wrap", ((0, 3, 0, 3), (9, 12, 9, 11))), ("clash", ((0, 3, 0, 3), (17, 20, 17, 20)))):
        n, na = 20, 16
        occ = np.zeros((n, n), dtype=bool)
        for r0, r1, c0, c1 in boxes:
            occ[r0:r1, c0:c1] = True
        x = rng.uniform(0, 1, (n, n))
        ang = np.linspace(0, 360, na, endpoint=False) + 0.3
        tg = geo.TargetGeometry(target=x.copy(), clip_to_circle=False)
        tg.segmentZ(0)
        tg.target = tg.array
        pg = geo.ProjectionGeometry(ang, "parallel", CUDA=False, occlusion=occ.copy())
        out[f"{tag}_occ"], out[f"{tag}_x"], out[f"{tag}_angles"] = occ, x, ang
        try:
            A2 = P2(tg, pg)
        except ValueError as exc:
            out[f"{tag}_error"] = np.array(str(exc))
            continue
        b = rng.uniform(0, 1, (n, na))
        out[f"{tag}_sino"] = A2.occ_sinogram
        out[f"{tag}_fwd"] = A2.forward(x.copy())
        out[f"{tag}_b"] = b
        out[f"{tag}_bwd"] = A2.backward(b.copy())
    np.savez_compressed(OUT / "occ2d.npz", **out)


def _ray_run(vam, tg, im, am, ab, ang, param, solver, rng):
    """Integrate a seeded field and deposit seeded energies through the reference's tracer."""
    geo = vam.geometry
    RT = vam.projector.pyTorchRayTrace
    pg = geo.ProjectionGeometry(ang, "ray_trace", CUDA=False, index_model=im, attenuation_model=am,
                                absorption_model=ab, ray_trace_method="eikonal", eikonal_parametrization=param,
                                ray_trace_ode_solver=solver, ray_trace_ray_config="parallel", inclination_angle=0.0,
                                ray_density=1)
    P = RT.PyTorchRayTracingPropagator(tg, pg)
    f = rng.uniform(0, 1, tg.array.shape)
    g = P.forward(f.copy())
    gin = rng.uniform(0, 1, g.shape).astype(np.float32)
    return f, np.asarray(g), gin, np.asarray(P.backward(gin.copy()))


def option_cases(vam):
    """Every selectable integrator x parametrisation of the reference's tracer on a graded-index grid
    medium, the analytic Luneburg-lens index (n_sur 1 and 1.2), the analytic homogeneous-ball
    attenuation, and the reference's dose metrics (calcVER / calcIPDR / calcPW / calcCV) on a seeded
    dose."""
    import torch

    geo, med = vam.geometry, vam.medium
    out = {}
    rng = np.random.default_rng(2024)
    n, nz = 12, 6
    tg = geo.TargetGeometry(target=rng.uniform(0, 1, (n, n, nz)))
    cv = tg.constructCoordVec()
    xg, yg, _ = np.meshgrid(*cv, indexing="ij")
    R = np.amax(cv[0])
    n_x = 1.30 + 0.05 * (xg ** 2 + yg ** 2) / R ** 2 + 0.01 * rng.uniform(-1, 1, xg.shape)
    alpha_x = 20.0 * (1 + 0.3 * rng.uniform(-1, 1, xg.shape))
    ang = np.linspace(0, 360, 5, endpoint=False)
    out["xv"], out["yv"], out["zv"] = cv
    out["n"], out["alpha"], out["angles"] = n_x, alpha_x, ang
    for param in ("physical_path_length", "canonical", "optical_path_length"):
        for solver in ("forward_symplectic_euler", "forward_euler", "leapfrog"):
            am = med.AttenuationModel(cv, type="interpolation", form="freeform", alpha_x=torch.as_tensor(alpha_x))
            if solver == "leapfrog":
                # the reference's leapfrog start-up step stores the index gradient into the float32 ray state
                # without a cast (pyTorchRayTrace.py:816-828): with an interpolated (float64) index field it
                # raises, so its leapfrog runs here through the analytic Luneburg lens (float32 gradient)
                im = med.IndexModel(cv, type="analytical", form="luneburg_lens", R=0.9, p=2, n_sur=1.2)
            else:
                im = med.IndexModel(cv, type="interpolation", form="freeform", n_x=torch.as_tensor(n_x))
            key = f"{param}__{solver}"
            f, g, gin, dose = _ray_run(vam, tg, im, am, am, ang, param, solver, rng)
            out[key + "_f"], out[key + "_fwd"], out[key + "_g"], out[key + "_bwd"] = f, g, gin, dose
    # analytic Luneburg lens (p = 2, radius 0.9 of the domain) with an absorbing cylinder
    for tag, n_sur in (("lune1", 1.0), ("lune12", 1.2)):
        im = med.IndexModel(cv, type="analytical", form="luneburg_lens", R=0.9, p=2, n_sur=n_sur)
        am = med.AttenuationModel(cv, type="analytical", form="homogeneous_cylinder", R=1, alpha_internal=15.0)
        f, g, gin, dose = _ray_run(vam, tg, im, am, am, ang, "physical_path_length", "forward_symplectic_euler", rng)
        out[tag + "_f"], out[tag + "_fwd"], out[tag + "_g"], out[tag + "_bwd"] = f, g, gin, dose
        out[tag + "_params"] = np.array([0.9, 2.0, n_sur])
    # analytic homogeneous ball attenuation (radius 0.8 of the domain) in a homogeneous index
    im = med.IndexModel(cv, type="analytical", form="homogeneous", n_sur=1.0)
    am = med.AttenuationModel(cv, type="analytical", form="homogeneous_ball", R=0.8, alpha_internal=25.0)
    f, g, gin, dose = _ray_run(vam, tg, im, am, am, ang, "physical_path_length", "forward_symplectic_euler", rng)
    out["ball_f"], out["ball_fwd"], out["ball_g"], out["ball_bwd"] = f, g, gin, dose
    out["ball_params"] = np.array([0.8, 25.0])
    # dose metrics on a seeded target and dose
    t = ellipses_target(20, 3, rng)
    tg2 = geo.TargetGeometry(target=t.copy())
    dose = rng.uniform(0, 1, t.shape) + 0.5 * t
    out["m_target"], out["m_dose"] = t, dose
    M = vam.metrics
    # (the reference's layerwise=True branches index a 2-D slice with the 3-D gel / void masks and raise
    # IndexError, metrics.py:78-90, 118-127, 158-166, so only the whole-volume values are stored)
    out["m_ver"], out["m_ipdr"], out["m_pw"] = M.calcVER(tg2, dose), M.calcIPDR(tg2, dose), M.calcPW(tg2, dose)
    out["m_cv"] = M.calcCV(tg2, dose)
    np.savez_compressed(OUT / "options.npz", **out)


def analytic_response_cases(vam):
    """BCLP with the reference's analytical generalised-logistic response model (evaluated in closed
    form, not by the interpolation table), p = 2 and p = 4 with weights."""
    geo = vam.geometry
    out = {}
    rng = np.random.default_rng(31)
    n, nz = 24, 2
    t = ellipses_target(n, nz, rng)
    # the analytical inverse map is -inf at a response of 0 (and the filtered initial sinogram NaN), so the
    # target's responses stay inside (0, 1), with no circle clip to zero the corners
    tgray = 0.05 + 0.9 * np.clip(t * 0.8 + 0.1 * rng.uniform(0, 1, t.shape), 0, 1)
    ang = np.linspace(0, 360, 18, endpoint=False)
    out["target"], out["angles"] = tgray, ang
    w = np.where(tgray > 0.15, 1.0, 0.5)
    out["weight"] = w
    for p, wt, lr in ((2, 1, 0.002), (4, w, 0.02)):
        rm = vam.response.ResponseModel(type="analytical", form="gen_log_fun", B=12, M=0.6)
        tg = geo.TargetGeometry(target=tgray.copy(), clip_to_circle=False)
        pg = geo.ProjectionGeometry(ang, "parallel", CUDA=False, attenuation_field=np.zeros((n, n, nz)))
        opts = refload.fresh_options(vam, method="BCLP", n_iter=4, p=p, q=1, eps=0.05, weight=wt, learning_rate=lr,
                                     response_model=rm, filter="ram-lak")
        sino, dose, mapped, logs = vam.optimize.optimize(tg, pg, opts, output="full")
        out[f"p{p}_sino"], out[f"p{p}_dose"], out[f"p{p}_mapped"] = sino.array, dose.array, mapped.array
        out[f"p{p}_loss"] = logs.loss
    np.savez_compressed(OUT / "analytic_bclp.npz", **out)


GROUPS = {"parallel": parallel_cases, "ray": ray_cases, "algebraic": algebraic_cases,
          "ray_autograd": ray_autograd_cases, "optim": optimizer_cases, "formats": format_cases,
          "vecgeom": vecgeom_cases, "occ2d": occ2d_cases, "options": option_cases,
          "analytic_bclp": analytic_response_cases}


def data_filter_cases(vam):
    """util.data's target filters (filterTarget, filterTargetBCLP) for every filter name and a 2-D and
    a 3-D input, and histogramEqualization, on seeded inputs."""
    D = vam.util.data
    rng = np.random.default_rng(77)
    out = {"x2": rng.uniform(0, 1, (24, 24)), "x3": rng.uniform(0, 1, (17, 17, 2)), "h": rng.normal(0, 1, (20, 12))}
    for name in ("ram-lak", "shepp-logan", "cosine", "hamming", "hanning"):
        for tag in ("x2", "x3"):
            out[f"bclp_{name}_{tag}"] = D.filterTargetBCLP(out[tag].copy(), name)
            out[f"target_{name}_{tag}"] = D.filterTarget(out[tag].copy(), name)
    out["histeq"] = D.histogramEqualization(out["h"].copy(), 8)
    np.savez_compressed(OUT / "datafilters.npz", **out)


GROUPS["datafilters"] = data_filter_cases


def main():
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", choices=sorted(GROUPS), help="regenerate only these fixture groups")
    args = ap.parse_args()
    warnings.simplefilter("ignore")
    vam = refload.load()
    for name, fn in GROUPS.items():
        if not args.only or name in args.only:
            fn(vam)
    for p in sorted(OUT.glob("*.npz")):
        print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main()
