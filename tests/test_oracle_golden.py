"""Pins the CPU oracle (oracle/vamoracle.c) against golden vectors produced by
the reference's own code (tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import relL2


@pytest.mark.parametrize("tag", ["even", "odd"])
def test_parallel_forward_backward_match_reference(golden, tag):
    P = golden["parallel"]
    b = O.parallel_forward(P[f"{tag}_x"], P[f"{tag}_angles"])
    assert np.array_equal(b, P[f"{tag}_fwd"]) or relL2(b, P[f"{tag}_fwd"]) < 1e-14
    x = O.parallel_backward_ref(P[f"{tag}_b"], P[f"{tag}_angles"])
    assert relL2(x, P[f"{tag}_bwd"]) < 1e-14


def test_occlusion_matches_reference(golden):
    P = golden["parallel"]
    occ, flag = O.occlusion_sinogram(P["occ_insert"], P["occ_angles"])
    ref = P["occ_sino"]
    assert np.array_equal(np.isnan(occ), np.isnan(ref))
    assert np.nanmax(np.abs(occ - ref)) == 0.0
    b = O.parallel_forward(P["occ_x"], P["occ_angles"], occlusion=(occ, flag))
    assert relL2(b, P["occ_fwd"]) < 1e-14
    x = O.parallel_backward_ref(P["occ_b"], P["occ_angles"], occlusion=(occ, flag))
    assert relL2(x, P["occ_bwd"]) < 1e-14


def test_2d_class_matches_3d_discretisation(golden):
    """The 2D class (Projector2DParallel.py:145-233) clips its input first and
    otherwise uses the same discretisation as the 3D class with nZ = 1."""
    P = golden["parallel"]
    x = O.clip_to_circle(P["p2_x"])
    b = O.parallel_forward(x[:, :, None], P["p2_angles"])[:, :, 0]
    assert relL2(b, P["p2_fwd"]) < 1e-14
    xb = O.parallel_backward_ref(P["p2_b"][:, :, None], P["p2_angles"])[:, :, 0]
    assert relL2(xb, P["p2_bwd"]) < 1e-14


def test_adjoint_is_transpose():
    rng = np.random.default_rng(0)
    ang = np.linspace(0, 360, 11, endpoint=False)
    x = rng.uniform(size=(20, 20, 2))
    y = rng.uniform(size=(20, 11, 2))
    for absn in (None, ("ray", 0.05, 8.0)):
        lhs = np.sum(O.parallel_forward(x, ang, absorption=absn) * y)
        rhs = np.sum(x * O.parallel_adjoint(y, ang, absorption=absn))
        assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_disk_sinogram_known_answer():
    """Sinogram of a centred uniform disk of radius rho is 2 sqrt(rho^2 - t^2)."""
    n, rho = 64, 20.0
    yy, xx = np.mgrid[:n, :n] - n // 2
    # supersampled disk so that bilinear sampling sees a smooth edge
    disk = np.zeros((n, n))
    for dy in np.linspace(-0.5, 0.5, 8, endpoint=False) + 1 / 16:
        for dx in np.linspace(-0.5, 0.5, 8, endpoint=False) + 1 / 16:
            disk += ((xx + dx) ** 2 + (yy + dy) ** 2 <= rho ** 2)
    disk /= 64
    b = O.parallel_forward(disk[:, :, None], np.array([0.0, 37.0, 90.0]))[:, :, 0]
    t = np.arange(n) - n // 2
    chord = 2 * np.sqrt(np.clip(rho ** 2 - t ** 2, 0, None))
    inner = np.abs(t) < rho - 2
    # pixelised disk vs the continuous chord: well under 1 % inside the disk
    assert np.max(np.abs(b[inner] - chord[inner, None]) / chord[inner, None]) < 0.01
    # 0 and 90 degrees sample mirror-image lattices of a symmetric disk
    assert np.allclose(b[:, 0], b[:, 2], rtol=0, atol=1e-12)


def test_ray_absorption_disk_known_answer():
    """Straight-ray transmission: with the per-ray weight exp(-alpha (s - s_entry)), s_entry =
    -sqrt(R^2 - t^2), a centred uniform disk of radius rho projects to
    exp(-alpha sqrt(R^2 - t^2)) 2 sinh(alpha sqrt(rho^2 - t^2)) / alpha."""
    n, rho, R, alpha = 128, 40.0, 56.0, 0.02
    yy, xx = np.mgrid[:n, :n] - n // 2
    disk = np.zeros((n, n))
    for dy in np.linspace(-0.5, 0.5, 8, endpoint=False) + 1 / 16:
        for dx in np.linspace(-0.5, 0.5, 8, endpoint=False) + 1 / 16:
            disk += ((xx + dx) ** 2 + (yy + dy) ** 2 <= rho ** 2)
    disk /= 64
    b = O.parallel_forward(disk[:, :, None], np.array([0.0, 37.0, 90.0, 211.0]), absorption=("ray", alpha, R))[:, :, 0]
    t = np.arange(n) - n // 2
    inner = np.abs(t) < rho - 2
    Lr, Lc = np.sqrt(np.clip(R ** 2 - t ** 2.0, 0, None)), np.sqrt(np.clip(rho ** 2 - t ** 2.0, 0, None))
    want = np.exp(-alpha * Lr) * 2 * np.sinh(alpha * Lc) / alpha
    assert np.max(np.abs(b[inner] - want[inner, None]) / want[inner, None]) < 0.01


def test_ray_oracle_matches_reference(golden):
    R = golden["raytrace"]
    for tag in ("r3", "r2"):
        xv, yv, zv = R[f"{tag}_xv"], R[f"{tag}_yv"], R[f"{tag}_zv"]
        x0, v0, _ = O.setup_rays_parallel(xv, yv, zv, R[f"{tag}_angles"])
        assert np.array_equal(x0, R[f"{tag}_x0"]) and np.array_equal(v0, R[f"{tag}_v0"])
        h, ms = R[f"{tag}_step"]
        grid = dict(xv=xv, yv=yv, zv=zv)
        a = R[f"{tag}_alpha"]
        kw = dict(step_size=h, max_num_step=int(ms), n_kind=1, n_grid=R[f"{tag}_n"], a_kind=3, a_grid=a, absorb=a)
        g, _ = O.ray_trace("integrate", grid, x0, v0, 1.0, f=R[f"{tag}_f"], **kw)
        assert relL2(g, R[f"{tag}_fwd"]) < 1e-6
        d, _ = O.ray_trace("deposit", grid, x0, v0, 1.0, g=R[f"{tag}_g"], **kw)
        assert relL2(d.squeeze(), R[f"{tag}_bwd"]) < 1e-6


def test_ray_oracle_analytic_medium(golden):
    import torch

    R = golden["raytrace"]
    xv, yv, zv = R["ha_xv"], R["ha_yv"], R["ha_zv"]
    x0, v0, _ = O.setup_rays_parallel(xv, yv, zv, R["ha_angles"])
    nsur, aval, _ = R["ha_params"]
    Rc = min((xv.max() - xv.min()) / 2, (yv.max() - yv.min()) / 2, (zv.max() - zv.min()) / 2)
    xg, yg, zg = np.meshgrid(xv, yv, zv, indexing="ij")
    r = torch.linalg.norm(torch.as_tensor(np.stack([xg.ravel(), yg.ravel()], 1)), dim=1).numpy()
    absorb = np.where(r < Rc, aval, 0.0).reshape(xg.shape)
    kw = dict(step_size=(xv[1] - xv[0]) / 2, max_num_step=3 * xv.size, n_kind=0, n_sur=nsur, a_kind=1,
              a_val=aval, a_R=Rc, absorb=absorb)
    g, _ = O.ray_trace("integrate", dict(xv=xv, yv=yv, zv=zv), x0, v0, 1.0, f=R["ha_f"], **kw)
    assert relL2(g, R["ha_fwd"]) < 1e-6
    d, _ = O.ray_trace("deposit", dict(xv=xv, yv=yv, zv=zv), x0, v0, 1.0, g=R["ha_g"], **kw)
    assert relL2(d, R["ha_bwd"]) < 1e-6


def test_ray_oracle_gradient_matches_reference_autograd(golden):
    """d<w, forward(f)>/df through the reference's autograd equals the oracle's deposit of w (the exact
    transpose), with the absorbing cylinder applied at the grid points."""
    import torch

    G = golden["ray_autograd"]
    xv, yv, zv = G["ag_xv"], G["ag_yv"], G["ag_zv"]
    x0, v0, _ = O.setup_rays_parallel(xv, yv, zv, G["ag_angles"])
    _, aval = G["ag_absorption"]
    Rc = min((xv.max() - xv.min()) / 2, (yv.max() - yv.min()) / 2, (zv.max() - zv.min()) / 2)
    xg, yg, zg = np.meshgrid(xv, yv, zv, indexing="ij")
    r = torch.linalg.norm(torch.as_tensor(np.stack([xg.ravel(), yg.ravel()], 1)), dim=1).numpy()
    absorb = np.where(r < Rc, aval, 0.0).reshape(xg.shape)
    kw = dict(step_size=(xv[1] - xv[0]) / 2, max_num_step=3 * xv.size, n_kind=1, n_grid=G["ag_n"], a_kind=3,
              a_grid=G["ag_alpha"], absorb=absorb)
    g, _ = O.ray_trace("integrate", dict(xv=xv, yv=yv, zv=zv), x0, v0, 1.0, f=G["ag_f"], **kw)
    assert relL2(g, G["ag_fwd"]) < 1e-6
    d, _ = O.ray_trace("deposit", dict(xv=xv, yv=yv, zv=zv), x0, v0, 1.0, g=G["ag_w"], **kw)
    assert relL2(d, G["ag_grad_f"]) < 1e-6


def test_host_filters_match_reference(golden):
    """The sinogram and OSMO target filters (numpy) against the reference's own outputs."""
    from vamtoolbox_b200.util import data as udata

    G = golden["optim"]
    for name in ("ram-lak", "shepp-logan", "cosine", "hamming", "hanning"):
        assert np.allclose(udata._get_fourier_filter(64, name)[:, 0], G["filt_" + name], rtol=0, atol=1e-12), name
    assert np.allclose(udata.filterSinogram(G["filt_sino_in"].copy(), "ram-lak"), G["filt_sino_ramlak"], atol=1e-12)
    assert np.allclose(udata.filterTargetOSMO(G["target"].copy(), "ram-lak"), G["filt_osmo"], atol=1e-12)


@pytest.mark.parametrize("tag", ["r3", "r2"])
def test_reference_propagation_matrix_is_its_forward(golden, tag):
    """The reference's recorded propagation matrix applied to f reproduces its ray-traced forward of f
    (absorption included): the fixture pins what the matrix means."""
    import scipy.sparse

    R = golden["raytrace"]
    A = scipy.sparse.coo_matrix((R[f"{tag}_mat_vals"], (R[f"{tag}_mat_rows"], R[f"{tag}_mat_cols"])),
                                shape=tuple(R[f"{tag}_mat_shape"])).tocsr()
    assert relL2(A @ R[f"{tag}_f"].reshape(-1), R[f"{tag}_fwd"]) < 1e-6


def test_occlusion_2d_digitised_matches_reference(golden):
    """The 2-D class's digitised occlusion (np.digitize bins, least occluded s per bin) and its shadowed
    forward and backward: the oracle's restatement gives the reference's outputs exactly."""
    G = golden["occ2d"]
    for tag in ("even", "odd", "wrap"):
        occ, x, ang = G[f"{tag}_occ"], G[f"{tag}_x"], G[f"{tag}_angles"]
        sino = O.occlusion_sinogram_2d(occ, ang)
        assert np.array_equal(sino, G[f"{tag}_sino"], equal_nan=True)
        assert np.isfinite(sino).any() and np.isnan(sino).any()
        assert relL2(O.parallel_forward_2d_occluded(x, ang, sino), G[f"{tag}_fwd"]) < 1e-14
        assert relL2(O.parallel_backward_2d_occluded(G[f"{tag}_b"], ang, sino), G[f"{tag}_bwd"]) < 1e-14
        if tag != "wrap":
            assert relL2(O.parallel_backward_2d_occluded(G[f"{tag}_b"], ang, sino, clipping=False),
                         G[f"{tag}_bwd_noclip"]) < 1e-14
        # the shadow matters: without it the forward differs
        free = O.parallel_forward(O.clip_to_circle(x)[:, :, None], ang)[:, :, 0]
        assert relL2(free, G[f"{tag}_fwd"]) > 0.1
    # the corner occluder of "clash" fills the last bin and wraps onto it: the reference raises
    with pytest.raises(ValueError, match="shape mismatch"):
        O.occlusion_sinogram_2d(G["clash_occ"], G["clash_angles"])
    assert "shape mismatch" in str(G["clash_error"])
