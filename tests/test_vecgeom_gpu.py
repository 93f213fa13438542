"""Vector-geometry (ASTRA-model) projector on the GPU (vam_vec_*) against the float64
oracle, and its place behind projectorconstructor / optimize for inclined rays."""
import numpy as np
import pytest
import torch

from oracle import vecgeom as V
from tests.conftest import relL2
from tests.test_vecgeom_golden import _smooth_phantom
from vamtoolbox_b200 import geometry, optimize, projectorconstructor
from vamtoolbox_b200.projector.Projector3DParallelCUDA import (Projector3DParallelCUDAAstra, VecPlan,
                                                               genVectorsAstra, parallel3d_vectors)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("incline,shape,n_ang", [(0.0, (40, 40, 12), 18), (15.0, (40, 40, 12), 18),
                                                  (-30.0, (32, 32, 20), 12), (55.0, (24, 24, 24), 10)])
def test_forward_backward_match_oracle(incline, shape, n_ang):
    rng = np.random.default_rng(4)
    vol = rng.random(shape)
    ang = np.linspace(0, 360, n_ang, endpoint=False) + 3.0
    vec = parallel3d_vectors(np.deg2rad(ang)) if incline == 0 else genVectorsAstra(ang, incline)
    n_u, n_v = shape[1], shape[2]
    plan = VecPlan(*shape, vec, n_u, n_v, "cuda")
    assert plan.info()["flat_forward"] == (incline == 0) and plan.info()["flat_backward"] == (incline == 0)
    f = plan.forward(torch.as_tensor(vol, dtype=torch.float32, device="cuda")).cpu().numpy()
    assert relL2(f, V.forward(vol, vec, n_u, n_v)) < 2e-5
    sino = rng.random((n_u, n_ang, n_v))
    b = plan.backward(torch.as_tensor(sino, dtype=torch.float32, device="cuda")).cpu().numpy()
    assert relL2(b, V.backward(sino, vec, shape)) < 2e-5


def test_dominant_z_axis_geometry():
    """Rays steeper than 45 degrees out of the plane step across z slices."""
    vec = genVectorsAstra(np.array([45.0, 135.0]), 70.0)
    assert (np.abs(vec[:, 2]) > np.abs(vec[:, :2]).max(1)).all()
    shape = (20, 20, 16)
    vol = _smooth_phantom(20, 16)
    plan = VecPlan(*shape, vec, 20, 16, "cuda")
    f = plan.forward(torch.as_tensor(vol, dtype=torch.float32, device="cuda")).cpu().numpy()
    assert relL2(f, V.forward(vol, vec, 20, 16)) < 2e-5


def _geo(n, nz, angles, **kw):
    tg = geometry.TargetGeometry(target=_smooth_phantom(n, nz) > 0.8)
    pg = geometry.ProjectionGeometry(angles, "parallel", CUDA=True, **kw)
    return tg, pg


def test_inclined_geometry_dispatches_to_vector_projector():
    tg, pg = _geo(32, 8, np.linspace(0, 360, 20, endpoint=False), inclination_angle=20.0)
    A = projectorconstructor.projectorconstructor(tg, pg)
    assert isinstance(A, Projector3DParallelCUDAAstra)
    x = np.array(tg.array, dtype=np.float64)
    b = A.forward(x)
    assert b.shape == (32, 20, 8) and b.dtype == np.float64
    ref = V.forward(x, genVectorsAstra(pg.angles, 20.0), 32, 8)
    assert relL2(b, ref) < 2e-5
    back = A.backward(b.copy())
    circle = np.asarray(__import__("vamtoolbox_b200.util.data", fromlist=["x"]).circle_inside_mask(32, 32))
    assert not back[~circle].any()                        # clipped to the inscribed circle
    tg2, pg2 = _geo(32, 8, np.linspace(0, 360, 20, endpoint=False))
    assert not isinstance(projectorconstructor.projectorconstructor(tg2, pg2), Projector3DParallelCUDAAstra)
    tg3, pg3 = _geo(32, 8, np.linspace(0, 360, 20, endpoint=False), parallel_model="astra")
    assert isinstance(projectorconstructor.projectorconstructor(tg3, pg3), Projector3DParallelCUDAAstra)


def test_forward_clips_input_in_place_and_backward_zeroes_zero_dose():
    tg, pg = _geo(24, 4, np.linspace(0, 180, 6, endpoint=False), inclination_angle=10.0)
    A = Projector3DParallelCUDAAstra(tg, pg)
    x = np.ones((24, 24, 4))
    A.forward(x)
    assert x[0, 0, 0] == 0 and x[12, 12, 0] == 1          # the reference clips its argument in place
    zd = np.zeros((24, 6, 4), dtype=bool)
    zd[3, 2, 1] = True
    pg.zero_dose_sino = zd
    b = np.ones((24, 6, 4))
    A.backward(b)
    assert b[3, 2, 1] == 0 and b[4, 2, 1] == 1


def test_device_tensors_stay_on_device():
    tg, pg = _geo(24, 4, np.linspace(0, 180, 6, endpoint=False), inclination_angle=10.0)
    A = Projector3DParallelCUDAAstra(tg, pg)
    x = torch.rand((24, 24, 4), device="cuda")
    b = A.forward(x)
    assert b.is_cuda and tuple(b.shape) == (24, 6, 4)
    assert A.backward(b).is_cuda


@pytest.mark.parametrize("method", ["BCLP", "CAL"])
def test_optimize_with_inclined_rays(method):
    tg, pg = _geo(32, 8, np.linspace(0, 360, 24, endpoint=False), inclination_angle=12.0)
    sino, recon, err = optimize.optimize(tg, pg, optimize.Options(method=method, n_iter=3, verbose=False))
    assert np.isfinite(np.asarray(sino.array)).all() and np.asarray(sino.array).shape == (32, 24, 8)


@pytest.mark.parametrize("shape,n_ang", [((40, 40), 36), ((33, 33), 17), ((64, 48), 20)])
def test_line2d_matches_oracle_and_is_a_transpose(shape, n_ang):
    from vamtoolbox_b200.projector.Projector2DParallelCUDA import Line2DPlan

    rng = np.random.default_rng(8)
    ang = np.sort(rng.uniform(0, 360, n_ang))
    ang[:4] = [0.0, 45.0, 90.0, 135.0]                     # axis-aligned and diagonal rays included
    n_t = shape[1]
    plan = Line2DPlan(*shape, ang, n_t, "cuda")
    img = rng.random(shape)
    f = plan.forward(img).cpu().numpy()
    assert relL2(f, V.line2d_forward(img, ang, n_t)) < 1e-5
    sino = rng.random((n_t, ang.size))
    b = plan.backward(sino).cpu().numpy()
    assert relL2(b, V.line2d_backward(sino, ang, shape)) < 1e-5
    lhs = float((f.astype(np.float64) * sino).sum())
    rhs = float((img * b.astype(np.float64)).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-6                # <A x, y> = <x, A^T y>


def test_line2d_dispatch():
    from vamtoolbox_b200.projector.Projector2DParallelCUDA import Projector2DParallelCUDAAstra

    tg = geometry.TargetGeometry(target=_smooth_phantom(48, 3) > 0.8)
    tg.segmentZ(1)
    pg = geometry.ProjectionGeometry(np.linspace(0, 180, 60, endpoint=False), "parallel", CUDA=True,
                                     parallel_model="astra")
    A = projectorconstructor.projectorconstructor(tg, pg)
    assert isinstance(A, Projector2DParallelCUDAAstra)
    x = np.ones((48, 48))
    b = A.forward(x)
    assert b.shape == (48, 60) and b.dtype == np.float64
    assert x[0, 0] == 0 and x[24, 24] == 1                 # the input is clipped in place
    back = A.backward(b.copy())
    from vamtoolbox_b200.util.data import circle_inside_mask
    assert back.shape == (48, 48) and not back[~circle_inside_mask(48, 48)].any()


@pytest.mark.parametrize("incline", [0.0, 15.0, 60.0])
def test_vec_adjoint_is_the_transpose(incline):
    shape = (28, 28, 16)
    ang = np.linspace(0, 360, 14, endpoint=False) + 2.0
    vec = parallel3d_vectors(np.deg2rad(ang)) if incline == 0 else genVectorsAstra(ang, incline)
    plan = VecPlan(*shape, vec, 28, 16, "cuda")
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.rand(shape, device="cuda", generator=g)
    y = torch.rand(plan.shape_sino, device="cuda", generator=g)
    lhs = float((plan.forward(x).double() * y.double()).sum())
    rhs = float((x.double() * plan.adjoint(y).double()).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


def test_autograd_vec_and_line2d():
    from vamtoolbox_b200 import autograd as AG
    from vamtoolbox_b200.projector.Projector2DParallelCUDA import Line2DPlan

    vec = genVectorsAstra(np.linspace(0, 360, 10, endpoint=False), 20.0)
    plan = VecPlan(20, 20, 12, vec, 20, 12, "cuda")
    x = torch.rand((20, 20, 12), device="cuda", requires_grad=True)
    w = torch.rand(plan.shape_sino, device="cuda")
    (AG.vec_forward(x, plan) * w).sum().backward()
    assert torch.allclose(x.grad, plan.adjoint(w), rtol=1e-5, atol=1e-6)

    lp = Line2DPlan(24, 24, np.linspace(0, 180, 16, endpoint=False), 24, "cuda")
    x2 = torch.rand((24, 24), device="cuda", dtype=torch.float32, requires_grad=True)
    w2 = torch.rand((24, 16), device="cuda")
    (AG.line2d_forward(x2, lp) * w2).sum().backward()
    assert torch.allclose(x2.grad, lp.backward(w2), rtol=1e-6, atol=1e-6)
    b2 = torch.rand((24, 16), device="cuda", requires_grad=True)
    w3 = torch.rand((24, 24), device="cuda")
    (AG.line2d_backward(b2, lp) * w3).sum().backward()
    assert torch.allclose(b2.grad, lp.forward(w3), rtol=1e-6, atol=1e-6)
    # a linear map: a central difference along a random direction equals the directional derivative
    d = torch.rand((24, 24), device="cuda")
    xd = x2.detach().double()
    fd = ((lp.forward((xd + 0.5 * d).float()).double() - lp.forward((xd - 0.5 * d).float()).double()) * w2).sum()
    assert abs(float(fd) - float((x2.grad * d).sum())) / abs(float(fd)) < 1e-4
