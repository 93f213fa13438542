"""Ray-tracing kernels (through the C ABI) against the reference's golden
vectors and the oracle.  Tolerance: relative L2 <= 1e-4 (float32 atomics)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.conftest import relL2

pytestmark = pytest.mark.gpu
TOL = 1e-4


def make_prop(R, tag, kind="grid"):
    from vamtoolbox_b200 import geometry, medium
    from vamtoolbox_b200.projector.pyTorchRayTrace import PyTorchRayTracingPropagator

    xv, yv, zv = R[f"{tag}_xv"], R[f"{tag}_yv"], R[f"{tag}_zv"]
    nz = zv.size
    tg = geometry.TargetGeometry(target=np.zeros((xv.size, yv.size, nz)) if nz > 1 else np.zeros((xv.size, yv.size)))
    cv = tg.constructCoordVec()
    assert all(np.array_equal(a, b) for a, b in zip(cv, (xv, yv, zv)))
    if kind == "grid":
        im = medium.IndexModel(cv, type="interpolation", form="freeform", n_x=torch.as_tensor(R[f"{tag}_n"]))
        am = medium.AttenuationModel(cv, type="interpolation", form="freeform", alpha_x=torch.as_tensor(R[f"{tag}_alpha"]))
    else:
        nsur, aval, _ = R["ha_params"]
        im = medium.IndexModel(cv, type="analytical", form="homogeneous", n_sur=float(nsur))
        am = medium.AttenuationModel(cv, type="analytical", form="homogeneous_cylinder", R=1, alpha_internal=float(aval))
    pg = geometry.ProjectionGeometry(R[f"{tag}_angles"], "ray_trace", CUDA=True, index_model=im, attenuation_model=am,
                                     absorption_model=am, ray_trace_method="eikonal",
                                     eikonal_parametrization="physical_path_length",
                                     ray_trace_ode_solver="forward_symplectic_euler", ray_trace_ray_config="parallel",
                                     inclination_angle=0.0, ray_density=1)
    return PyTorchRayTracingPropagator(tg, pg)


@pytest.mark.parametrize("tag", ["r3", "r2"])
def test_integrate_deposit_match_reference_golden(golden, tag):
    R = golden["raytrace"]
    P = make_prop(R, tag)
    assert np.array_equal(P.plan.x0.numpy(), R[f"{tag}_x0"])
    g = P.forward(R[f"{tag}_f"])
    assert relL2(g, R[f"{tag}_fwd"]) < TOL
    d = P.backward(R[f"{tag}_g"])
    assert relL2(d, R[f"{tag}_bwd"]) < TOL


def test_analytic_medium_matches_reference_golden(golden):
    R = golden["raytrace"]
    P = make_prop(R, "ha", kind="analytic")
    assert relL2(P.forward(R["ha_f"]), R["ha_fwd"]) < TOL
    assert relL2(P.backward(R["ha_g"]), R["ha_bwd"]) < TOL


def test_integrate_is_transpose_of_deposit(golden):
    R = golden["raytrace"]
    P = make_prop(R, "r3")
    rng = np.random.default_rng(2)
    f = torch.as_tensor(rng.uniform(size=P.plan.grid_shape), device="cuda", dtype=torch.float32)
    w = torch.as_tensor(rng.uniform(size=P.plan.num_rays), device="cuda", dtype=torch.float32)
    lhs = float((P.forward_t(f).double() * w.double()).sum())
    rhs = float((f.double() * P.backward_t(w).double()).sum())
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


def test_active_rays_at_cap_reported(golden):
    R = golden["raytrace"]
    P = make_prop(R, "r3")
    P.forward(R["r3_f"])
    # the reference logged 265/360 rays active at its 36-step cap for this case
    assert P.plan.active_at_cap() == 265


def test_grad_alpha_matches_finite_differences(golden):
    R = golden["raytrace"]
    P = make_prop(R, "r3")
    rng = np.random.default_rng(4)
    f = torch.as_tensor(rng.uniform(size=P.plan.grid_shape), device="cuda", dtype=torch.float32)
    w = torch.as_tensor(rng.uniform(size=P.plan.num_rays), device="cuda", dtype=torch.float32)
    grad = torch.zeros(P.plan.grid_shape, device="cuda", dtype=torch.float32)
    P.plan.grad_alpha(f, w, grad_att=grad)
    from vamtoolbox_b200 import medium

    cv = [R["r3_xv"], R["r3_yv"], R["r3_zv"]]
    base = R["r3_alpha"]
    for k in range(3):
        d = rng.standard_normal(base.shape)
        h = 1e-2 * np.abs(base).max()

        def L(alpha):
            am = medium.AttenuationModel(cv, type="interpolation", form="freeform", alpha_x=torch.as_tensor(alpha))
            P.plan.bind_medium(P.proj_geo.index_model, am, P.proj_geo.absorption_model)
            return float((P.forward_t(f).double() * w.double()).sum())

        fd = (L(base + h * d) - L(base - h * d)) / (2 * h)
        an = float((grad.double().cpu() * torch.as_tensor(d)).sum())
        assert abs(fd - an) <= 2e-2 * abs(fd) + 1e-6, (fd, an)
    P.plan.bind_medium(P.proj_geo.index_model, P.proj_geo.attenuation_model, P.proj_geo.absorption_model)


def test_angle_shards_reproduce_the_full_run(golden):
    """Projectors built on angle shards of the geometry (the multi-GPU split, run here one after the
    other on one GPU) trace the full run's rays: their integrals are the full run's sinogram rows at
    ray_indices, bit for bit, and their deposits sum to the full deposit (float32 atomics: 1e-5)."""
    from vamtoolbox_b200.distributed import angle_range, ray_indices, shard_angles
    from vamtoolbox_b200.projector.pyTorchRayTrace import PyTorchRayTracingPropagator

    R = golden["raytrace"]
    P = make_prop(R, "r3")
    rng = np.random.default_rng(6)
    f = torch.as_tensor(rng.uniform(size=P.plan.grid_shape), device="cuda", dtype=torch.float32)
    w = torch.as_tensor(rng.uniform(size=P.plan.num_rays), device="cuda", dtype=torch.float32)
    full_rows = P.forward_t(f).cpu().numpy()
    full_dose = P.backward_t(w).double()
    n_ang = len(P.proj_geo.angles)
    n_det = P.plan.num_rays // (n_ang * P.plan.grid_shape[2])
    dose = torch.zeros_like(full_dose)
    for rank in range(2):
        Pr = PyTorchRayTracingPropagator(P.target_geo, shard_angles(P.proj_geo, 2, rank))
        idx = ray_indices(n_det, n_ang, P.plan.grid_shape[2], *angle_range(n_ang, 2, rank))
        assert np.array_equal(Pr.forward_t(f).cpu().numpy(), full_rows[idx])
        dose += Pr.backward_t(w[torch.as_tensor(idx, device="cuda")]).double()
    assert float((dose - full_dose).norm() / full_dose.norm()) < 1e-5


def test_integrate_is_bitwise_repeatable(golden):
    """The integrate has no atomics (one thread per ray, fixed sample order): repeated calls, and a
    call after a deposit has reused the plan's scratch field, give identical bits."""
    R = golden["raytrace"]
    P = make_prop(R, "r3")
    f = torch.as_tensor(np.random.default_rng(8).uniform(size=P.plan.grid_shape), device="cuda", dtype=torch.float32)
    first = P.forward_t(f).clone()
    for _ in range(3):
        assert torch.equal(P.forward_t(f), first)
    P.backward_t(torch.ones(P.plan.num_rays, device="cuda"))
    assert torch.equal(P.forward_t(f), first)


def test_trajectory_cache_bitwise_and_invalidated(golden):
    """With the trajectory cache (rays traced once, each step's position and attenuance kept) integrate
    and deposit stream the records instead of re-tracing: the integrate gives the tracing kernel's bits,
    the deposit its sums up to the order of its float32 atomics, the same count of rays active at the
    cap; a new medium invalidates the cache, and a cache over its byte limit is refused without changing
    the results."""
    R = golden["raytrace"]
    P = make_prop(R, "r3")
    plan = P.plan
    rng = np.random.default_rng(11)
    f = torch.as_tensor(rng.uniform(size=plan.grid_shape), device="cuda", dtype=torch.float32)
    w = torch.as_tensor(rng.uniform(size=plan.num_rays), device="cuda", dtype=torch.float32)
    w[::7] = 0.0  # rays with no energy deposit nothing
    g0, d0 = plan.integrate(f).clone(), plan.deposit(w).clone()
    cap0 = plan.active_at_cap()
    # not even one warp of rays fits: refused, the plan keeps tracing
    assert not plan.prepare_trajectories(limit_bytes=plan.trajectory_bytes(32) - 1)
    assert torch.equal(plan.integrate(f), g0)
    # a prefix of the rays (a multiple of 32) cached, the rest traced: the same results
    assert plan.num_rays > 96
    assert plan.prepare_trajectories(limit_bytes=plan.trajectory_bytes(plan.num_rays // 2))
    m = plan.cached_rays
    assert 0 < m < plan.num_rays and m % 32 == 0
    assert torch.equal(plan.integrate(f), g0)
    assert plan.active_at_cap() == cap0
    assert relL2(plan.deposit(w).cpu().numpy(), d0.cpu().numpy()) < 1e-5
    assert plan.active_at_cap() == cap0
    assert plan.prepare_trajectories()
    assert plan.cached_rays == plan.num_rays
    assert plan.has_trajectories
    for _ in range(2):
        assert torch.equal(plan.integrate(f), g0)
        assert plan.active_at_cap() == cap0
        assert relL2(plan.deposit(w).cpu().numpy(), d0.cpu().numpy()) < 1e-5
        assert plan.active_at_cap() == cap0
    # a changed medium: the cache is dropped from use and the results follow the new medium
    P2 = make_prop(R, "r3")
    am_scale = 1.7
    from vamtoolbox_b200 import medium

    cv = P2.target_geo.constructCoordVec() if hasattr(P2, "target_geo") else None
    im = medium.IndexModel(cv, type="interpolation", form="freeform", n_x=torch.as_tensor(R["r3_n"]))
    am = medium.AttenuationModel(cv, type="interpolation", form="freeform",
                                 alpha_x=torch.as_tensor(R["r3_alpha"] * am_scale))
    plan.bind_medium(im, am, am)
    P2.plan.bind_medium(im, am, am)
    assert not plan.has_trajectories
    assert torch.equal(plan.integrate(f), P2.plan.integrate(f))
    assert relL2(plan.deposit(w).cpu().numpy(), P2.plan.deposit(w).cpu().numpy()) < 1e-5
    plan.drop_trajectories()
