"""Parallel-beam kernels (through the C ABI) against the oracle and the
reference's golden vectors.  Tolerance: relative L2 <= 1e-5 (float32 kernels
vs the reference's float64), dot test <= 1e-6 relative."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.conftest import relL2

pytestmark = pytest.mark.gpu
TOL = 1e-5


def plan_for(shape, angles):
    from vamtoolbox_b200.projector.Projector3DParallel import ParallelPlan

    return ParallelPlan(shape[0], shape[1], shape[2], angles)


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device="cuda")


@pytest.mark.parametrize("tag", ["even", "odd"])
def test_forward_backward_match_reference_golden(golden, tag):
    P = golden["parallel"]
    x, ang = P[f"{tag}_x"], P[f"{tag}_angles"]
    p = plan_for(x.shape, ang)
    b = p.forward(dev(x)).cpu().numpy()
    assert relL2(b, P[f"{tag}_fwd"]) < TOL
    xb = p.backward_ref(dev(P[f"{tag}_b"])).cpu().numpy()
    assert relL2(xb, P[f"{tag}_bwd"]) < TOL


def test_occlusion_matches_reference_golden(golden):
    P = golden["parallel"]
    p = plan_for(P["occ_x"].shape, P["occ_angles"])
    p.set_occlusion(P["occ_insert"])
    occ = p.occlusion_sinogram().cpu().numpy()
    ref = P["occ_sino"]
    assert np.array_equal(np.isnan(occ), np.isnan(ref))
    assert np.nanmax(np.abs(occ - ref)) == 0.0
    assert relL2(p.forward(dev(P["occ_x"])).cpu().numpy(), P["occ_fwd"]) < TOL
    assert relL2(p.backward_ref(dev(P["occ_b"])).cpu().numpy(), P["occ_bwd"]) < TOL


@pytest.mark.parametrize("shape,na", [((32, 32, 8), 24), ((33, 33, 5), 17), ((40, 40, 1), 30),
                                      ((24, 24, 12), 9), ((48, 48, 64), 12), ((20, 20, 3), 360)])
def test_against_oracle_shapes(shape, na):
    rng = np.random.default_rng(sum(shape) + na)
    ang = np.sort(rng.uniform(0, 360, na))
    ang[0] = 0.0
    x = rng.uniform(0, 1, shape)
    b = rng.uniform(0, 1, (shape[0], na, shape[2]))
    p = plan_for(shape, ang)
    assert relL2(p.forward(dev(x)).cpu().numpy(), O.parallel_forward(x, ang)) < TOL
    assert relL2(p.backward_ref(dev(b)).cpu().numpy(), O.parallel_backward_ref(b, ang)) < TOL
    assert relL2(p.adjoint(dev(b)).cpu().numpy(), O.parallel_adjoint(b, ang)) < TOL


def test_exact_angles_and_binary_target():
    """Multiples of 90 degrees put samples on integer coordinates (floor == ceil)."""
    n = 64
    yy, xx = np.mgrid[:n, :n] - n / 2
    x = ((xx ** 2 + yy ** 2) < 20 ** 2).astype(float)[:, :, None] * np.ones((1, 1, 4))
    ang = np.array([0.0, 45.0, 90.0, 180.0, 270.0, 359.5])
    p = plan_for(x.shape, ang)
    assert relL2(p.forward(dev(x)).cpu().numpy(), O.parallel_forward(x, ang)) < TOL
    bb = O.parallel_forward(x, ang)
    assert relL2(p.backward_ref(dev(bb)).cpu().numpy(), O.parallel_backward_ref(bb, ang)) < TOL


@pytest.mark.parametrize("absn", [None, "ray", "mask"])
def test_adjoint_dot_product(absn):
    rng = np.random.default_rng(3)
    shape, na = (36, 36, 8), 20
    ang = np.linspace(0, 360, na, endpoint=False) + 0.3
    p = plan_for(shape, ang)
    mask = None
    if absn == "ray":
        p.set_absorption("ray", alpha_per_px=0.03, radius_px=15.0)
        oabs = ("ray", 0.03, 15.0)
    elif absn == "mask":
        mask = rng.uniform(0.2, 1.0, shape[:2])
        p.set_absorption("mask", mask=mask)
        oabs = ("mask", mask)
    else:
        oabs = None
    x = rng.uniform(0, 1, shape)
    y = rng.uniform(0, 1, (shape[0], na, shape[2]))
    Ax = p.forward(dev(x)).double()
    Aty = p.adjoint(dev(y)).double()
    lhs = float((Ax * dev(y).double()).sum())
    rhs = float((dev(x).double() * Aty).sum())
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)
    # signed inputs: error relative to the sum of magnitudes
    xs, ys = dev(rng.standard_normal(shape)), dev(rng.standard_normal((shape[0], na, shape[2])))
    a1 = p.forward(xs).double() * ys.double()
    a2 = xs.double() * p.adjoint(ys).double()
    assert abs(float(a1.sum() - a2.sum())) <= 1e-6 * float(a1.abs().sum())
    assert relL2(Ax.cpu().numpy(), O.parallel_forward(x, ang, absorption=oabs)) < TOL
    assert relL2(p.backward_ref(dev(y)).cpu().numpy(), O.parallel_backward_ref(y, ang, absorption=oabs)) < TOL


def test_occlusion_adjoint_is_transpose(golden):
    P = golden["parallel"]
    p = plan_for(P["occ_x"].shape, P["occ_angles"])
    p.set_occlusion(P["occ_insert"])
    rng = np.random.default_rng(5)
    x = rng.standard_normal(P["occ_x"].shape)
    y = rng.standard_normal(P["occ_fwd"].shape)
    lhs = float((p.forward(dev(x)).double() * dev(y).double()).sum())
    rhs = float((dev(x).double() * p.adjoint(dev(y)).double()).sum())
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


def test_mask_matches_reference_mask(golden):
    from vamtoolbox_b200 import geometry

    P = golden["parallel"]
    px, a, R = P["mask_params"]
    tg = geometry.TargetGeometry(target=np.ones((24, 24, 2)))
    pg = geometry.ProjectionGeometry(np.array([0.0]), "parallel", projector_pixel_size=px, absorption_coeff=a,
                                     container_radius=R)
    pg.calcAbsorptionMask(tg)
    assert np.array_equal(pg.absorption_mask[:, :, 0], P["mask"])


def test_projector_class_numpy_roundtrip(golden):
    from vamtoolbox_b200 import geometry
    from vamtoolbox_b200.projector.Projector3DParallel import Projector3DParallel

    P = golden["parallel"]
    x, ang = P["even_x"], P["even_angles"]
    tg = geometry.TargetGeometry(target=x.copy(), clip_to_circle=False)
    pg = geometry.ProjectionGeometry(ang, "parallel", CUDA=True)
    A = Projector3DParallel(tg, pg)
    b = A.forward(x)
    assert isinstance(b, np.ndarray) and b.dtype == np.float64 and b.shape == P["even_fwd"].shape
    assert relL2(b, P["even_fwd"]) < TOL
    assert relL2(A.backward(P["even_b"]), P["even_bwd"]) < TOL
    t = A.forward(torch.as_tensor(x, device="cuda", dtype=torch.float32))
    assert t.is_cuda and t.dtype == torch.float32


def test_deterministic_gather_kernels():
    rng = np.random.default_rng(11)
    shape, ang = (40, 40, 16), np.linspace(0, 180, 33)
    x, y = dev(rng.uniform(size=shape)), dev(rng.uniform(size=(40, 33, 16)))
    p = plan_for(shape, ang)
    for f, a in ((p.forward, x), (p.backward_ref, y), (p.adjoint, y)):
        assert torch.equal(f(a), f(a))


def test_bad_inputs_raise():
    from vamtoolbox_b200._lib import VamError

    p = plan_for((16, 16, 4), np.linspace(0, 180, 8))
    with pytest.raises(ValueError):
        p.forward(torch.zeros((16, 16, 5), device="cuda"))
    with pytest.raises(TypeError):
        p.forward(torch.zeros((16, 16, 4), device="cuda", dtype=torch.float64))
    with pytest.raises(VamError):
        p.set_absorption("ray", alpha_per_px=float("nan"), radius_px=3.0)


FAST_CASES = [
    ((32, 32, 128), np.linspace(0, 360, 24, endpoint=False)),     # even N, all angles paired, VZ=4
    ((33, 33, 256), np.linspace(0, 360, 20, endpoint=False)),     # odd N, paired, VZ=8
    ((30, 30, 128), None),                                        # unpaired random angles
    ((28, 28, 192), np.concatenate([np.linspace(0, 180, 7, endpoint=False), [200.0, 380.0]])),  # mixed
]


@pytest.mark.parametrize("shape,ang", FAST_CASES)
@pytest.mark.parametrize("absn", [None, "mask", "ray"])
def test_fast_paths_against_oracle(shape, ang, absn):
    rng = np.random.default_rng(shape[2] + shape[0])
    if ang is None:
        ang = np.sort(rng.uniform(0, 360, 17))
    x = rng.uniform(0, 1, shape)
    b = rng.uniform(0, 1, (shape[0], ang.size, shape[2]))
    p = plan_for(shape, ang)
    oabs = None
    if absn == "mask":
        m = rng.uniform(0.3, 1.0, shape[:2])
        p.set_absorption("mask", mask=m)
        oabs = ("mask", m)
    elif absn == "ray":
        p.set_absorption("ray", alpha_per_px=0.04, radius_px=shape[0] / 2 - 1.5)
        oabs = ("ray", 0.04, shape[0] / 2 - 1.5)
    assert relL2(p.forward(dev(x)).cpu().numpy(), O.parallel_forward(x, ang, absorption=oabs)) < TOL
    assert relL2(p.backward_ref(dev(b)).cpu().numpy(), O.parallel_backward_ref(b, ang, absorption=oabs)) < TOL
    assert relL2(p.adjoint(dev(b)).cpu().numpy(), O.parallel_adjoint(b, ang, absorption=oabs)) < TOL
    # dot test <Ax, y> = <x, A^T y>
    Ax = p.forward(dev(x)).double()
    lhs = float((Ax * dev(b).double()).sum())
    rhs = float((dev(x).double() * p.adjoint(dev(b)).double()).sum())
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)


@pytest.mark.parametrize("absn", [None, "ray"])
def test_adjoint_without_weight_table(absn):
    """The on-the-fly matched transpose (used when the table is not built or is too large)."""
    rng = np.random.default_rng(9)
    shape, ang = (30, 30, 128), np.linspace(0, 360, 18, endpoint=False) + 0.7
    p = plan_for(shape, ang)
    p.adj_table_limit_bytes = 0
    oabs = None
    if absn == "ray":
        p.set_absorption("ray", alpha_per_px=0.04, radius_px=13.0)
        oabs = ("ray", 0.04, 13.0)
    b = rng.uniform(0, 1, (30, 18, 128))
    assert relL2(p.adjoint(dev(b)).cpu().numpy(), O.parallel_adjoint(b, ang, absorption=oabs)) < TOL
    assert not p._adj_ready


TUNINGS = [dict(forward_vz=fv, backward_vz=bv, backward_batch=bb, adjoint_vz=av, adjoint_table=at, backward_table=bt)
           for fv, (bv, bb, bt), (av, at) in [(4, (4, 1, 0), (4, 1)), (8, (8, 1, 0), (8, 1)), (4, (4, 2, 0), (4, 0)),
                                              (8, (8, 2, 0), (8, 0)), (4, (4, 4, 0), (8, 1)), (1, (1, 1, 0), (1, 0)),
                                              (8, (8, 2, 1), (8, 1))]]


@pytest.mark.parametrize("tuning", TUNINGS, ids=lambda t: "-".join(str(v) for v in t.values()))
@pytest.mark.parametrize("absn", [None, "ray"])
def test_every_launch_shape_matches_oracle(tuning, absn):
    """Each launch shape the autotuner can pick (vector width, angle batch, table) gives the oracle's result,
    including an angle count that is not a multiple of the batch and paired + unpaired angles."""
    rng = np.random.default_rng(77)
    shape = (29, 29, 256)
    ang = np.concatenate([np.linspace(0, 360, 14, endpoint=False), [7.3, 101.9, 250.1]])
    x = rng.uniform(0, 1, shape)
    b = rng.uniform(0, 1, (shape[0], ang.size, shape[2]))
    p = plan_for(shape, ang)
    oabs = None
    if absn == "ray":
        p.set_absorption("ray", alpha_per_px=0.05, radius_px=12.5)
        oabs = ("ray", 0.05, 12.5)
    p.set_tuning(tuning)
    if tuning["backward_table"]:
        assert p.prepare_backward()
    got = p.get_tuning()
    assert {k: got[k] for k in tuning} == tuning
    assert relL2(p.forward(dev(x)).cpu().numpy(), O.parallel_forward(x, ang, absorption=oabs)) < TOL
    assert relL2(p.backward_ref(dev(b)).cpu().numpy(), O.parallel_backward_ref(b, ang, absorption=oabs)) < TOL
    assert relL2(p.adjoint(dev(b)).cpu().numpy(), O.parallel_adjoint(b, ang, absorption=oabs)) < TOL


def test_autotune_caches_winner(tmp_path, monkeypatch):
    monkeypatch.setenv("VAMTOOLBOX_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    from vamtoolbox_b200 import autotune as AT

    p = plan_for((40, 40, 128), np.linspace(0, 180, 30, endpoint=False))
    first = p.autotune()
    d = AT._load(str(tmp_path / "tune.json"))
    key = AT.problem_key(p)
    assert d[key]["tuning"] == first and set(d[key]["ms"]) == {"forward", "backward", "adjoint"}
    q = plan_for((40, 40, 128), np.linspace(0, 180, 30, endpoint=False))
    assert q.autotune() == first
    with pytest.raises(Exception):
        q.set_tuning({"backward_batch": 3})


@pytest.mark.parametrize("n,na", [(40, 30), (33, 17), (128, 180), (257, 90)])
@pytest.mark.parametrize("absn", [None, "mask", "ray"])
@pytest.mark.parametrize("path", ["tiles", "generic"])
def test_single_slice_paths_against_oracle(n, na, absn, path):
    """2-D slices: the shared-memory tile kernels (default) and the generic kernels both match the oracle."""
    rng = np.random.default_rng(n + na)
    ang = np.sort(rng.uniform(0, 360, na))
    ang[0] = 0.0
    x = rng.uniform(0, 1, (n, n, 1))
    b = rng.uniform(0, 1, (n, na, 1))
    p = plan_for(x.shape, ang)
    oabs = None
    if absn == "mask":
        m = rng.uniform(0.3, 1.0, (n, n))
        p.set_absorption("mask", mask=m)
        oabs = ("mask", m)
    elif absn == "ray":
        p.set_absorption("ray", alpha_per_px=0.02, radius_px=n / 2 - 1.5)
        oabs = ("ray", 0.02, n / 2 - 1.5)
    if path == "generic":
        p.set_tuning({"forward_vz": 1, "backward_vz": 1, "adjoint_vz": 1})
    else:
        p.set_tuning({"forward_vz": 4, "backward_vz": 4})  # tiles at every size
    assert relL2(p.forward(dev(x)).cpu().numpy(), O.parallel_forward(x, ang, absorption=oabs)) < TOL
    assert relL2(p.backward_ref(dev(b)).cpu().numpy(), O.parallel_backward_ref(b, ang, absorption=oabs)) < TOL


@pytest.mark.parametrize("nz", [1, 8])
def test_ray_absorption_disk_known_answer(nz):
    """Per-ray absorption, centred uniform disk of radius rho inside a container of radius R: the
    weight exp(-alpha (s - s_entry)), s_entry = -sqrt(R^2 - t^2), integrates over the disk's chord
    to b(t) = exp(-alpha sqrt(R^2 - t^2)) 2 sinh(alpha sqrt(rho^2 - t^2)) / alpha (straight-ray
    transmission); with alpha -> 0 it is the chord 2 sqrt(rho^2 - t^2)."""
    from vamtoolbox_b200.projector.Projector3DParallel import ParallelPlan

    n, rho, R, alpha = 128, 40.0, 56.0, 0.02
    yy, xx = np.mgrid[:n, :n] - n // 2
    disk = np.zeros((n, n))
    for dy in np.linspace(-0.5, 0.5, 8, endpoint=False) + 1 / 16:
        for dx in np.linspace(-0.5, 0.5, 8, endpoint=False) + 1 / 16:
            disk += ((xx + dx) ** 2 + (yy + dy) ** 2 <= rho ** 2)
    disk /= 64
    angles = np.array([0.0, 37.0, 90.0, 211.0])
    p = ParallelPlan(n, n, nz, angles)
    p.set_absorption("ray", alpha_per_px=alpha, radius_px=R)
    x = torch.as_tensor(np.repeat(disk[:, :, None], nz, axis=2), dtype=torch.float32, device="cuda").contiguous()
    b = p.forward(x).cpu().numpy().astype(np.float64)
    t = np.arange(n) - n // 2
    inner = np.abs(t) < rho - 2
    Lr, Lc = np.sqrt(np.clip(R ** 2 - t ** 2.0, 0, None)), np.sqrt(np.clip(rho ** 2 - t ** 2.0, 0, None))
    want = np.exp(-alpha * Lr) * 2 * np.sinh(alpha * Lc) / alpha
    rel = np.abs(b[inner] - want[inner, None, None]) / want[inner, None, None]
    assert rel.max() < 0.01
    for k in range(1, nz):
        assert np.array_equal(b[:, :, k], b[:, :, 0])


def _proj2d(x, ang, occ=None):
    from vamtoolbox_b200 import geometry
    from vamtoolbox_b200.projector.Projector2DParallel import Projector2DParallel

    tg = geometry.TargetGeometry(target=x.copy())
    pg = geometry.ProjectionGeometry(ang, "parallel", CUDA=True, occlusion=None if occ is None else occ.copy())
    return Projector2DParallel(tg, pg)


@pytest.mark.parametrize("tag", ["even", "odd", "wrap"])
def test_occlusion_2d_matches_reference_golden(golden, tag):
    """The 2-D class's digitised occlusion on the device: the occlusion sinogram bit for bit (float64
    minima, NaN pattern), the shadowed forward and backprojection within the projector tolerance; "wrap"
    has occluders below the first detector bin at some angles (the reference's shifted bin pairing)."""
    G = golden["occ2d"]
    A = _proj2d(G[f"{tag}_x"], G[f"{tag}_angles"], G[f"{tag}_occ"])
    sino = A.occ_sinogram
    assert np.array_equal(sino, G[f"{tag}_sino"], equal_nan=True)
    assert relL2(A.forward(G[f"{tag}_x"].copy()), G[f"{tag}_fwd"]) < TOL
    assert relL2(A.backward(G[f"{tag}_b"].copy()), G[f"{tag}_bwd"]) < TOL
    if tag != "wrap":
        assert relL2(A.backward(G[f"{tag}_b"].copy(), clipping=False), G[f"{tag}_bwd_noclip"]) < TOL


def test_occlusion_2d_raises_where_the_reference_raises(golden):
    G = golden["occ2d"]
    with pytest.raises(ValueError, match="shape mismatch"):
        _proj2d(G["clash_x"], G["clash_angles"], G["clash_occ"])
    with pytest.raises(ValueError, match="zero-size array"):
        _proj2d(G["even_x"], G["even_angles"], np.zeros_like(G["even_occ"]))


def test_occlusion_2d_adjoint_is_transpose(golden):
    G = golden["occ2d"]
    n, ang = G["wrap_x"].shape[0], G["wrap_angles"]
    p = plan_for((n, n, 1), ang)
    p.set_occlusion_2d(G["wrap_occ"])
    rng = np.random.default_rng(6)
    x, y = rng.standard_normal((n, n, 1)), rng.standard_normal((n, ang.size, 1))
    lhs = float((p.forward(dev(x)).double() * dev(y).double()).sum())
    rhs = float((dev(x).double() * p.adjoint(dev(y)).double()).sum())
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


@pytest.mark.parametrize("n", [40, 363])
def test_backward_without_clipping_matches_oracle(n):
    """backward(b, clipping=False) of the 2-D class without occlusion: every pixel, inside the circle or
    not, against the oracle's unclipped np.interp backprojection."""
    rng = np.random.default_rng(n)
    ang = np.linspace(0, 360, 90, endpoint=False) + 0.25
    A = _proj2d(rng.uniform(size=(n, n)), ang)
    b = rng.uniform(size=(n, ang.size))
    got = A.backward(b.copy(), clipping=False)
    ref = O.parallel_backward_2d_occluded(b, ang, np.full((n, ang.size), np.nan), clipping=False)
    assert relL2(got, ref) < TOL
    assert np.abs(got[~O.circle_mask((n, n))]).max() > 0  # pixels outside the circle are not clipped
    assert relL2(A.backward(b.copy()), O.clip_to_circle(ref)) < TOL


def test_released_plan_is_reused_reset():
    """A plan whose ParallelPlan object was released is handed to the next plan of the same geometry with no
    absorption, no occlusion and the default launch shapes; its results equal a fresh plan's."""
    import gc

    from vamtoolbox_b200.projector import Projector3DParallel as P3

    P3.clear_plan_pool()
    shape, ang = (40, 40, 64), np.linspace(0, 360, 24, endpoint=False)
    rng = np.random.default_rng(12)
    x, b = rng.uniform(size=shape), rng.uniform(size=(40, 24, 64))
    p = plan_for(shape, ang)
    ref_fwd, ref_bwd = p.forward(dev(x)).cpu().numpy(), p.backward_ref(dev(b)).cpu().numpy()
    first = p.handle.value
    p.set_absorption("ray", alpha_per_px=0.05, radius_px=15.0)
    p.set_occlusion(np.zeros(shape))
    p.set_tuning({"forward_vz": 1, "backward_table": 0})
    del p
    gc.collect()
    q = plan_for(shape, ang)
    assert q.handle.value == first
    assert q.get_tuning() == P3._DEFAULT_TUNING
    assert np.array_equal(q.forward(dev(x)).cpu().numpy(), ref_fwd)
    assert np.array_equal(q.backward_ref(dev(b)).cpu().numpy(), ref_bwd)
    other = plan_for((40, 40, 64), ang + 1.0)  # different angles: a new plan
    assert other.handle.value != first
    q.close()
    P3.clear_plan_pool()


@pytest.mark.parametrize("ny,nx,na", [(256, 256, 90), (384, 384, 45), (363, 363, 60), (258, 258, 37)])
@pytest.mark.parametrize("mode", ["none", "mask", "ray"])
def test_tma_staged_slice_forward_matches_plain_loads_and_oracle(ny, nx, na, mode):
    """The 2-D tile forward stages its footprint boxes with TMA tensor copies; an image whose rows are not a
    multiple of 16 bytes, one at an address off a 16-byte boundary, and a masked image are first copied into
    the plan's padded image.  Every route gives the plain-load staging's sums bit for bit, those are the
    oracle's, and the plan records no timeout."""
    rng = np.random.default_rng(ny * nx)
    ang = np.linspace(0, 360, na, endpoint=False) + 0.4
    x = rng.uniform(0, 1, (ny, nx, 1))
    p = plan_for((ny, nx, 1), ang)
    oabs = None
    if mode == "mask":
        m = rng.uniform(0.2, 1.0, (ny, nx))
        p.set_absorption("mask", mask=m)
        oabs = ("mask", m)
    elif mode == "ray":
        p.set_absorption("ray", alpha_per_px=0.01, radius_px=min(nx, ny) / 2.0)
        oabs = ("ray", 0.01, min(nx, ny) / 2.0)
    aligned = dev(x)
    buf = torch.zeros(ny * nx + 1, device="cuda")
    buf[1:] = aligned.reshape(-1)
    misaligned = buf[1:].reshape(ny, nx, 1)  # 4 bytes past a 16-byte boundary
    assert aligned.data_ptr() % 16 == 0 and misaligned.data_ptr() % 16 == 4
    a = p.forward(aligned).cpu().numpy()
    b = p.forward(misaligned).cpu().numpy()
    p.set_tuning({"forward_tma": 0})
    c = p.forward(aligned).cpu().numpy()
    d = p.forward(misaligned).cpu().numpy()
    assert np.array_equal(a, b) and np.array_equal(a, c) and np.array_equal(a, d)
    assert relL2(a, O.parallel_forward(x, ang, absorption=oabs)) < TOL
    assert p.status() == 0


@pytest.mark.parametrize("shape,na,mode", [((64, 64, 256), 90, None), ((63, 63, 128), 47, "mask"),
                                           ((40, 40, 512), 33, None), ((34, 34, 64), 40, None),
                                           ((37, 37, 200), 25, "mask"), ((30, 30, 12), 19, None)])
def test_backprojection_table_bitwise_and_oracle(shape, na, mode):
    """The backprojection from the plan's 2 x 2 block bin table, with four and with eight slices per lane,
    gives the computed-bin kernel's sums bit for bit, and the oracle's within float32 tolerance: odd widths
    (partial blocks and tiles), several z chunks and partial ones (nZ not a multiple of 128 or 256), angle
    counts that are not multiples of 32 (partial entry chunks), mask absorption."""
    rng = np.random.default_rng(sum(shape) + na)
    ang = np.linspace(0, 360, na, endpoint=False) + 0.7
    p = plan_for(shape, ang)
    oabs = None
    if mode == "mask":
        m = rng.uniform(0.2, 1.0, shape[:2])
        p.set_absorption("mask", mask=m)
        oabs = ("mask", m)
    b = rng.uniform(0, 1, (shape[0], na, shape[2]))
    p.set_tuning({"backward_vz": 8, "backward_table": 0})
    computed = p.backward_ref(dev(b))
    assert p.prepare_backward()
    for vz in (4, 8):
        p.set_tuning({"backward_table": 1, "backward_vz": vz})
        tabled = p.backward_ref(dev(b))
        assert torch.equal(computed, tabled), vz
    assert relL2(tabled.cpu().numpy(), O.parallel_backward_ref(b, ang, absorption=oabs)) < TOL
    assert p.status() == 0


@pytest.mark.parametrize("shape,na,absn,vz", [((33, 33, 192), 29, None, 6), ((24, 24, 384), 36, "ray", 6),
                                              ((30, 30, 192), 40, "mask", 6), ((28, 28, 160), 31, None, 5),
                                              ((26, 26, 320), 24, "mask", 5), ((22, 22, 160), 30, "ray", 5)])
def test_six_slice_lanes_bitwise(shape, na, absn, vz):
    """Six / five slices per lane (a float4 and a float2 / a float per lane: 192- / 160-slice chunks fill
    every lane where 256-slice ones would not) give the eight-slice kernels' sums bit for bit: the forward
    (paired and unpaired angles, per-ray and mask absorption) and the block-table backprojection, and the
    oracle's."""
    rng = np.random.default_rng(sum(shape) + na)
    ang = np.linspace(0, 360, na, endpoint=False) + 0.9
    x = rng.uniform(0, 1, shape)
    b = rng.uniform(0, 1, (shape[0], na, shape[2]))
    p = plan_for(shape, ang)
    oabs = None
    if absn == "ray":
        p.set_absorption("ray", alpha_per_px=0.04, radius_px=shape[0] / 2 - 1.0)
        oabs = ("ray", 0.04, shape[0] / 2 - 1.0)
    elif absn == "mask":
        m = rng.uniform(0.2, 1.0, shape[:2])
        p.set_absorption("mask", mask=m)
        oabs = ("mask", m)
    p.set_tuning({"forward_vz": 8})
    f8 = p.forward(dev(x))
    p.set_tuning({"forward_vz": vz})
    f6 = p.forward(dev(x))
    p.set_tuning({"forward_vz": 0})
    f0 = p.forward(dev(x))
    assert torch.equal(f6, f8) and torch.equal(f0, f8)
    assert relL2(f6.cpu().numpy(), O.parallel_forward(x, ang, absorption=oabs)) < TOL
    if absn != "ray":
        p.set_tuning({"backward_vz": 8, "backward_table": 0})
        computed = p.backward_ref(dev(b))
        assert p.prepare_backward()
        p.set_tuning({"backward_vz": 0, "backward_table": 1})  # automatic: six / five slices per lane
        assert torch.equal(p.backward_ref(dev(b)), computed)
    assert p.status() == 0
