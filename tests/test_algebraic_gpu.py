"""The propagation matrix of the ray tracer (vam_ray_record_*) and the algebraic propagator
(vam_csr_spmm) against the reference's buildPropagationMatrix and PyTorchAlgebraicPropagator outputs,
and against this package's own integrate / deposit kernels."""
import numpy as np
import pytest
import scipy.sparse
import torch

from tests.conftest import relL2
from tests.test_raytrace_gpu import make_prop

pytestmark = pytest.mark.gpu


def dense(rows, cols, vals, shape):
    return scipy.sparse.coo_matrix((vals, (rows, cols)), shape=shape).toarray()


@pytest.mark.parametrize("tag", ["r3", "r2"])
def test_propagation_matrix_matches_reference(golden, tag):
    R = golden["raytrace"]
    P = make_prop(R, tag)
    M = P.buildPropagationMatrix()
    assert tuple(M.shape) == tuple(R[f"{tag}_mat_shape"])
    ref = dense(R[f"{tag}_mat_rows"], R[f"{tag}_mat_cols"], R[f"{tag}_mat_vals"], tuple(R[f"{tag}_mat_shape"]))
    assert relL2(M.toarray(), ref) < 1e-4


@pytest.mark.parametrize("tag", ["r3", "r2"])
def test_propagation_matrix_is_integrate_and_its_transpose_deposit(golden, tag):
    R = golden["raytrace"]
    P = make_prop(R, tag)
    P.output_torch_tensor = True
    A = P.buildPropagationMatrix().to_sparse_csr()
    rng = np.random.default_rng(5)
    f = torch.as_tensor(rng.uniform(size=P.plan.grid_shape), dtype=torch.float32, device="cuda")
    g = torch.as_tensor(rng.uniform(size=P.plan.num_rays), dtype=torch.float32, device="cuda")
    Af = (A @ f.reshape(-1, 1)).reshape(-1)
    assert relL2(Af.cpu().numpy(), P.forward_t(f).cpu().numpy()) < 1e-5
    ATg = (A.t() @ g.reshape(-1, 1)).reshape(-1)
    assert relL2(ATg.cpu().numpy(), P.backward_t(g).reshape(-1).cpu().numpy()) < 1e-5


def test_algebraic_propagator_matches_reference(golden, tmp_path):
    """A one-layer matrix loaded from a SciPy .npz file and z-tiled over a three-layer volume."""
    from vamtoolbox_b200 import geometry
    from vamtoolbox_b200.projectorconstructor import projectorconstructor

    R, G = golden["raytrace"], golden["algebraic"]
    M = scipy.sparse.coo_matrix((R["r2_mat_vals"], (R["r2_mat_rows"], R["r2_mat_cols"])),
                                shape=tuple(R["r2_mat_shape"]))
    path = tmp_path / "propagation_matrix.npz"
    scipy.sparse.save_npz(path, M.tocsr())
    tg = geometry.TargetGeometry(target=G["x"].copy())
    pg = geometry.ProjectionGeometry(np.linspace(0, 360, 5, endpoint=False), "algebraic", CUDA=True,
                                     loading_path_for_matrix=str(path))
    A = projectorconstructor(tg, pg)
    assert A.z_tiling == int(G["z_tiling"]) == 3
    assert relL2(A.forward(G["x"]), G["fwd"]) < 1e-5
    assert relL2(A.backward(G["b"]), G["bwd"]) < 1e-5
    # deterministic
    assert np.array_equal(A.forward(G["x"]), A.forward(G["x"]))


def test_algebraic_propagator_from_built_matrix(golden):
    """A matrix handed over directly (no file), from this package's own tracer: forward equals integrate."""
    from vamtoolbox_b200 import geometry
    from vamtoolbox_b200.projector.pyTorchAlgebraicPropagation import PyTorchAlgebraicPropagator

    R = golden["raytrace"]
    P = make_prop(R, "r3")
    tg = geometry.TargetGeometry(target=np.zeros(P.plan.grid_shape))
    A = PyTorchAlgebraicPropagator(tg, None, matrix=P.buildPropagationMatrix())
    f = np.random.default_rng(2).uniform(size=P.plan.grid_shape)
    assert relL2(A.forward(f), P.forward(f)) < 1e-5
    with pytest.raises(Exception):
        PyTorchAlgebraicPropagator(geometry.TargetGeometry(target=np.zeros((5, 5, 5))), None,
                                   matrix=P.buildPropagationMatrix())


@pytest.mark.parametrize("ztile", [1, 3, 4, 128, 132])
def test_csr_kernel_tilings(ztile):
    """vam_csr_spmm on every path (one column, narrow, 16-byte vectors, more than 128 columns) against a
    float64 reference product."""
    from vamtoolbox_b200 import _lib

    rng = np.random.default_rng(ztile)
    A = scipy.sparse.random(300, 200, density=0.05, random_state=ztile, format="csr", dtype=np.float64)
    A.data = A.data.astype(np.float32).astype(np.float64)
    X = rng.uniform(-1, 1, (200, ztile)).astype(np.float32)
    ref = A @ X.astype(np.float64)
    rp = torch.as_tensor(A.indptr.astype(np.int64), device="cuda")
    ci = torch.as_tensor(A.indices.astype(np.int32), device="cuda")
    va = torch.as_tensor(A.data.astype(np.float32), device="cuda")
    x = torch.as_tensor(X, device="cuda").contiguous()
    y = torch.full((300, ztile), float("nan"), device="cuda")
    _lib.call("vam_csr_spmm", 300, _lib.ptr(rp), _lib.ptr(ci), _lib.ptr(va), _lib.ptr(x), ztile, _lib.ptr(y),
              _lib.stream_ptr())
    assert relL2(y.cpu().numpy(), ref) < 1e-6


def test_algebraic_bclp_device_engine_matches_host_engine():
    """BCLP through the algebraic propagator on the fused device engine (its CSR products captured with
    the dose pass and update in one graph) gives the reference's host loop result."""
    from vamtoolbox_b200 import geometry, medium
    from vamtoolbox_b200.optimize import Options, optimize
    from vamtoolbox_b200.projector.pyTorchRayTrace import PyTorchRayTracingPropagator

    n, na = 24, 18
    rng = np.random.default_rng(4)
    t = np.zeros((n, n))
    y, x = np.mgrid[:n, :n] - (n - 1) / 2
    t[(x / 8.0) ** 2 + (y / 6.0) ** 2 <= 1] = 1.0
    tg = geometry.TargetGeometry(target=t)
    cv = tg.constructCoordVec()
    im = medium.IndexModel(cv, type="interpolation", form="homogeneous")
    am = medium.AttenuationModel(cv, type="analytical", form="homogeneous_cylinder", R=1, alpha_internal=1e-3)
    pg = geometry.ProjectionGeometry(np.linspace(0, 180, na, endpoint=False), "ray_trace", CUDA=True, index_model=im,
                                     attenuation_model=am, absorption_model=am,
                                     eikonal_parametrization="physical_path_length",
                                     ray_trace_ode_solver="forward_symplectic_euler", ray_trace_ray_config="parallel")
    P = PyTorchRayTracingPropagator(tg, pg)
    P.output_torch_tensor = True
    import scipy.sparse
    import tempfile, os

    M = P.buildPropagationMatrix()
    idx = M.coalesce().indices().cpu().numpy()
    S = scipy.sparse.csr_matrix((M.coalesce().values().cpu().numpy(), (idx[0], idx[1])), shape=tuple(M.shape))
    out = {}
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "P.npz")
        scipy.sparse.save_npz(path, S)
        for engine in ("device", "host"):
            pga = geometry.ProjectionGeometry(np.linspace(0, 180, na, endpoint=False), "algebraic", CUDA=False,
                                              loading_path_for_matrix=path)
            tga = geometry.TargetGeometry(target=t)
            sino, dose, mapped, logs = optimize(tga, pga, Options(method="BCLP", n_iter=5, p=2, q=1, eps=0.1,
                                                                  learning_rate=1e-2, filter=None, engine=engine),
                                                output="full")
            out[engine] = (np.asarray(sino.array), np.asarray(dose.array), logs.loss.copy())
    assert relL2(out["device"][0], out["host"][0]) < 1e-4
    assert relL2(out["device"][1], out["host"][1]) < 1e-4
    assert np.allclose(out["device"][2], out["host"][2], rtol=1e-4)
