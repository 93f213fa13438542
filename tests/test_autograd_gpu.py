"""autograd through the hand-written adjoints: gradcheck-style comparisons
against central finite differences along random directions."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_parallel_forward_gradient_is_matched_adjoint():
    from vamtoolbox_b200.autograd import parallel_forward
    from vamtoolbox_b200.projector.Projector3DParallel import ParallelPlan

    rng = np.random.default_rng(0)
    shape, ang = (32, 32, 128), np.linspace(0, 360, 20, endpoint=False)
    p = ParallelPlan(*shape, ang)
    x = torch.as_tensor(rng.uniform(size=shape), device="cuda", dtype=torch.float32, ).requires_grad_(True)
    w = torch.as_tensor(rng.standard_normal((32, 20, 128)), device="cuda", dtype=torch.float32)
    loss = (parallel_forward(x, p) * w).sum()
    loss.backward()
    for k in range(8):
        d = torch.as_tensor(rng.standard_normal(shape), device="cuda", dtype=torch.float32)
        h = 1e-2
        with torch.no_grad():
            fp = (p.forward((x + h * d).contiguous()).double() * w.double()).sum()
            fm = (p.forward((x - h * d).contiguous()).double() * w.double()).sum()
        fd = float((fp - fm) / (2 * h))
        an = float((x.grad.double() * d.double()).sum())
        assert abs(fd - an) <= 2e-4 * (abs(fd) + 1e-3), (fd, an)


def test_parallel_bclp_loss_gradient_matches_finite_differences():
    """Sinogram gradient of a BCLP-style loss through R1^T (central FD, h = 1e-3)."""
    from vamtoolbox_b200.autograd import parallel_adjoint
    from vamtoolbox_b200.projector.Projector3DParallel import ParallelPlan

    rng = np.random.default_rng(1)
    shape, na = (24, 24, 128), 16
    p = ParallelPlan(*shape, np.linspace(0, 360, na, endpoint=False))
    tgt = torch.as_tensor((rng.uniform(size=shape) > 0.5).astype(np.float32), device="cuda")
    g = torch.as_tensor(rng.uniform(0, 0.05, (24, na, 128)), device="cuda", dtype=torch.float32).requires_grad_(True)

    def loss_fn(gg):
        dose = parallel_adjoint(gg, p)
        mapped = torch.sigmoid(12 * (dose - 0.6))
        eb = (mapped - tgt).abs() - 0.05
        return (torch.relu(eb) ** 2).sum().double()

    L = loss_fn(g)
    L.backward()
    for k in range(4):
        d = torch.as_tensor(rng.standard_normal(g.shape), device="cuda", dtype=torch.float32)
        h = 1e-3
        with torch.no_grad():
            fd = float((loss_fn(g + h * d) - loss_fn(g - h * d)) / (2 * h))
        an = float((g.grad.double() * d.double()).sum())
        assert abs(fd - an) <= 2e-2 * abs(fd) + 1e-6, (fd, an)


def test_ray_integrate_gradients():
    from vamtoolbox_b200 import geometry, medium
    from vamtoolbox_b200.autograd import ray_integrate
    from vamtoolbox_b200.projector.pyTorchRayTrace import RayPlan

    rng = np.random.default_rng(2)
    n = 14
    tg = geometry.TargetGeometry(target=np.zeros((n, n, 6)))
    cv = tg.constructCoordVec()
    xg, yg, _ = np.meshgrid(*cv, indexing="ij")
    im = medium.IndexModel(cv, type="interpolation", form="freeform",
                           n_x=torch.as_tensor(1.4 + 0.05 * (xg ** 2 + yg ** 2) / np.amax(cv[0]) ** 2))
    alpha0 = 25.0 * (1 + 0.2 * rng.uniform(-1, 1, xg.shape))
    am = medium.AttenuationModel(cv, type="interpolation", form="freeform", alpha_x=torch.as_tensor(alpha0))
    ab = medium.AbsorptionModel(cv, type="analytical", form="homogeneous_cylinder", alpha_internal=10.0)
    plan = RayPlan(cv, np.linspace(0, 360, 6, endpoint=False), im, am, ab)
    f = torch.as_tensor(rng.uniform(size=plan.grid_shape), device="cuda", dtype=torch.float32).requires_grad_(True)
    alpha = torch.as_tensor(alpha0, device="cuda", dtype=torch.float32).requires_grad_(True)
    w = torch.as_tensor(rng.uniform(size=plan.num_rays), device="cuda", dtype=torch.float32)
    L = (ray_integrate(f, plan, alpha, im, am, ab) * w).sum()
    L.backward()
    with torch.no_grad():
        for k in range(3):
            d = torch.as_tensor(rng.standard_normal(plan.grid_shape), device="cuda", dtype=torch.float32)
            # linear in f: FD is exact up to float32 rounding
            fd = float(((ray_integrate(f + d, plan, alpha, im, am, ab) - ray_integrate(f - d, plan, alpha, im, am, ab))
                        .double() * w.double()).sum() / 2)
            an = float((f.grad.double() * d.double()).sum())
            assert abs(fd - an) <= 1e-4 * abs(fd) + 1e-6, (fd, an)
            h = 0.5
            fd = float(((ray_integrate(f, plan, alpha + h * d, im, am, ab)
                         - ray_integrate(f, plan, alpha - h * d, im, am, ab)).double() * w.double()).sum() / (2 * h))
            an = float((alpha.grad.double() * d.double()).sum())
            assert abs(fd - an) <= 2e-2 * abs(fd) + 1e-5, (fd, an)


def test_ray_gradients_match_reference_autograd(golden):
    """Gradients of L = <w, integrate(f)> w.r.t. f and the attenuation grid, against autograd through the
    reference's own PyTorch ray tracer (float64 fields there, float32 here).  Tolerances: relative L2
    1e-4 for d/df (a linear map: the deposit), 2e-3 for d/dalpha (float32 exp / suffix sums of the
    attenuance against the reference's float64 autograd graph)."""
    from tests.conftest import relL2
    from vamtoolbox_b200 import geometry, medium
    from vamtoolbox_b200.autograd import ray_integrate
    from vamtoolbox_b200.projector.pyTorchRayTrace import RayPlan

    G = golden["ray_autograd"]
    cv = [G["ag_xv"], G["ag_yv"], G["ag_zv"]]
    tg = geometry.TargetGeometry(target=np.zeros((cv[0].size, cv[1].size, cv[2].size)))
    assert all(np.array_equal(a, b) for a, b in zip(tg.constructCoordVec(), cv))
    im = medium.IndexModel(cv, type="interpolation", form="freeform", n_x=torch.as_tensor(G["ag_n"]))
    am = medium.AttenuationModel(cv, type="interpolation", form="freeform", alpha_x=torch.as_tensor(G["ag_alpha"]))
    R_abs, a_abs = G["ag_absorption"]
    ab = medium.AttenuationModel(cv, type="analytical", form="homogeneous_cylinder", R=float(R_abs),
                                 alpha_internal=float(a_abs))
    plan = RayPlan(cv, G["ag_angles"], im, am, ab)
    f = torch.as_tensor(G["ag_f"], device="cuda", dtype=torch.float32).requires_grad_(True)
    alpha = torch.as_tensor(G["ag_alpha"], device="cuda", dtype=torch.float32).requires_grad_(True)
    w = torch.as_tensor(G["ag_w"], device="cuda", dtype=torch.float32)
    g = ray_integrate(f, plan, alpha, im, am, ab)
    assert relL2(g.detach().cpu().numpy(), G["ag_fwd"]) < 1e-4
    L = (g * w).sum()
    L.backward()
    assert abs(float(L) - float(G["ag_L"])) <= 1e-4 * abs(float(G["ag_L"]))
    assert relL2(f.grad.cpu().numpy(), G["ag_grad_f"]) < 1e-4
    assert relL2(alpha.grad.cpu().numpy(), G["ag_grad_alpha"]) < 2e-3
