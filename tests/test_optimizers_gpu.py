"""Optimizers through the public API vs the reference's own optimizer runs
(tests/golden/optim.npz, float64 numpy) and device engine vs host engine."""
import numpy as np
import pytest

from tests.conftest import relL2

pytestmark = pytest.mark.gpu


def geo(target, angles):
    from vamtoolbox_b200 import geometry

    return geometry.TargetGeometry(target=target.copy()), geometry.ProjectionGeometry(angles, "parallel", CUDA=True)


def opts(**kw):
    from vamtoolbox_b200.optimize import Options

    return Options(**kw)


def counts_close(a, b, tg):
    n = np.sum(tg.gel_inds) + np.sum(tg.void_inds)
    return np.all(np.abs(np.asarray(a) - np.asarray(b)) * n <= 1.0 + 1e-9)


@pytest.mark.parametrize("engine", ["device", "host"])
def test_cal_matches_reference(golden, engine):
    from vamtoolbox_b200.optimize import optimize

    O = golden["optim"]
    tg, pg = geo(O["target"], O["angles"])
    s, r, e = optimize(tg, pg, opts(method="CAL", n_iter=5, learning_rate=0.4, d_h=0.5, sigmoid=0.01, engine=engine))
    assert relL2(s.array, O["cal_sino"]) < 1e-4
    assert relL2(r.array, O["cal_recon"]) < 1e-4
    assert counts_close(e, O["cal_err"], tg)


@pytest.mark.parametrize("engine", ["device", "host"])
def test_osmo_matches_reference(golden, engine):
    from vamtoolbox_b200.optimize import optimize

    O = golden["optim"]
    tg, pg = geo(O["target"], O["angles"])
    s, r, e = optimize(tg, pg, opts(method="OSMO", n_iter=4, d_h=0.8, d_l=0.7, filter="ram-lak", engine=engine))
    assert relL2(s.array, O["osmo_sino"]) < 1e-4
    assert relL2(r.array, O["osmo_recon"]) < 1e-4
    assert counts_close(e, O["osmo_err"], tg)


def test_fbp_matches_reference(golden):
    from vamtoolbox_b200.optimize import optimize

    O = golden["optim"]
    tg, pg = geo(O["target"], O["angles"])
    s, r, e = optimize(tg, pg, opts(method="FBP", n_iter=1, filter="ram-lak"))
    assert relL2(s.array, O["fbp_sino"]) < 1e-5
    assert relL2(r.array, O["fbp_recon"]) < 1e-5
    assert counts_close(e[:1], O["fbp_err"][:1], tg)


@pytest.mark.parametrize("engine", ["device", "host"])
def test_bclp_matches_reference(golden, engine):
    from vamtoolbox_b200.optimize import optimize
    from vamtoolbox_b200.response import ResponseModel

    O = golden["optim"]
    tg, pg = geo(O["bclp_target"], O["angles"])
    rm = ResponseModel(B=12, M=0.6)
    assert np.array_equal(rm.interp_map_0, O["resp_map"]) and np.array_equal(rm.interp_dmapdf_0, O["resp_dmap"])
    sino, dose, mapped, logs = optimize(tg, pg, opts(method="BCLP", n_iter=4, p=2, q=1, eps=0.05, learning_rate=0.002,
                                                     response_model=rm, filter="ram-lak", engine=engine), output="full")
    assert relL2(sino.array, O["bclp_sino"]) < 1e-4
    assert relL2(dose.array, O["bclp_dose"]) < 1e-4
    assert relL2(mapped.array, O["bclp_mapped"]) < 1e-4
    assert np.allclose(logs.loss, O["bclp_loss"], rtol=1e-4)
    norms = np.stack([logs.l0, logs.l1, logs.l2, logs.lf, logs.l0_eps0, logs.l1_eps0, logs.l2_eps0, logs.lf_eps0])
    assert np.all(np.abs(norms[0] - O["bclp_norms"][0]) <= 1)  # voxel counts
    assert np.allclose(norms[1:4], O["bclp_norms"][1:4], rtol=1e-3, atol=1e-5)
    assert np.allclose(norms[5:], O["bclp_norms"][5:], rtol=1e-3, atol=1e-5)


def test_bclp_step_interface_matches_reference(golden):
    """The reference's step interface of BCLPNorm (getLossGrad / getLoss / callback / updateVariables /
    evaluateNormMetrics: the calls an external optimizer makes), driven the way the reference's own
    gradientDescent drives it, reproduces the reference's BCLP run; the state is computed once per
    iteration index, so a second getLoss at the same index does not project again."""
    from vamtoolbox_b200.optimizer.BCLP import BCLPNorm
    from vamtoolbox_b200.response import ResponseModel

    O = golden["optim"]
    tg, pg = geo(O["bclp_target"], O["angles"])
    b = BCLPNorm(tg, pg, opts(method="BCLP", n_iter=4, p=2, q=1, eps=0.05, learning_rate=0.002,
                              response_model=ResponseModel(B=12, M=0.6), filter="ram-lak"))
    g = b.checkSinogramShape(b.host_g0(), desired_shape="flattened")
    for _ in range(4):
        g = b.imposeSinogramConstraints(g - b.learning_rate * b.getLossGrad(g))
        dose_before = b.dose
        b.getLoss(g)
        assert b.dose is dose_before  # same iteration index: nothing recomputed
        b.callback(g)
    b.updateVariables(g)
    b.evaluateNormMetrics()
    assert relL2(b.checkSinogramShape(g, desired_shape="cylindrical"), O["bclp_sino"]) < 1e-4
    assert relL2(b.dose, O["bclp_dose"]) < 1e-4
    assert relL2(b.mapped_dose, O["bclp_mapped"]) < 1e-4
    L = b.logs
    assert np.allclose(L.loss, O["bclp_loss"], rtol=1e-4)
    norms = np.stack([L.l0, L.l1, L.l2, L.lf, L.l0_eps0, L.l1_eps0, L.l2_eps0, L.lf_eps0])
    assert np.all(np.abs(norms[0] - O["bclp_norms"][0]) <= 1)  # voxel counts
    assert np.allclose(norms[1:4], O["bclp_norms"][1:4], rtol=1e-3, atol=1e-5)
    assert np.allclose(norms[5:], O["bclp_norms"][5:], rtol=1e-3, atol=1e-5)


def test_pm_runs_and_tracks_reference(golden):
    from vamtoolbox_b200.optimize import optimize

    O = golden["optim"]
    tg, pg = geo(O["target"], O["angles"])
    s, r, e = optimize(tg, pg, opts(method="PM", n_iter=3, d_h=0.8, d_l=0.6, rho_1=1, rho_2=1, p=2))
    assert relL2(s.array, O["pm_sino"]) < 1e-3
    assert np.isfinite(e[0])


def test_bclp_graph_equals_eager():
    from vamtoolbox_b200.optimize import Options
    from vamtoolbox_b200.optimizer import BCLP
    from vamtoolbox_b200 import geometry

    rng = np.random.default_rng(1)
    t = np.clip(rng.uniform(size=(32, 32, 8)), 0, 1)
    out = []
    for graph in (True, False):
        tg = geometry.TargetGeometry(target=t.copy())
        pg = geometry.ProjectionGeometry(np.linspace(0, 360, 24, endpoint=False), "parallel")
        b = BCLP.BCLPNorm(tg, pg, Options(method="BCLP", n_iter=6, learning_rate=1e-3))
        out.append((b.gradientDescentDevice(graph=graph), b.logs.loss.copy()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_options_do_not_leak_between_instances():
    a = opts(method="CAL", learning_rate=0.4)
    b = opts(method="CAL")
    assert a.learning_rate == 0.4 and b.learning_rate == 0.01


@pytest.mark.parametrize("engine", ["device", "host"])
def test_bclp_p4_weighted_matches_reference(golden, engine):
    """BCLP with the fourth-power band norm and per-voxel weights (1 inside the target, 0.5 outside)."""
    from vamtoolbox_b200.optimize import optimize
    from vamtoolbox_b200.response import ResponseModel

    O = golden["optim"]
    tg, pg = geo(O["bclp_target"], O["angles"])
    sino, dose, mapped, logs = optimize(tg, pg, opts(method="BCLP", n_iter=4, p=4, q=1, eps=0.05,
                                                     weight=O["bclp4_weight"], learning_rate=0.02,
                                                     response_model=ResponseModel(B=12, M=0.6), filter="ram-lak",
                                                     engine=engine), output="full")
    assert relL2(sino.array, O["bclp4_sino"]) < 1e-4
    assert relL2(dose.array, O["bclp4_dose"]) < 1e-4
    assert np.allclose(logs.loss, O["bclp4_loss"], rtol=1e-4)


@pytest.mark.parametrize("engine", ["device", "host"])
def test_cal_single_slice_matches_reference(golden, engine):
    """CAL on a 2-D target (stored as n x n x 1, as the reference does)."""
    from vamtoolbox_b200.optimize import optimize

    O = golden["optim"]
    tg, pg = geo(O["cal2d_target"], O["angles"])
    s, r, e = optimize(tg, pg, opts(method="CAL", n_iter=5, learning_rate=0.4, d_h=0.5, sigmoid=0.01, engine=engine))
    assert relL2(np.reshape(s.array, O["cal2d_sino"].shape), O["cal2d_sino"]) < 1e-4
    assert relL2(np.reshape(r.array, O["cal2d_recon"].shape), O["cal2d_recon"]) < 1e-4
    assert counts_close(e, O["cal2d_err"], tg)


def test_device_filters_match_reference(golden):
    """cuFFT versions of the sinogram and OSMO target filters against the reference's numpy outputs."""
    import torch

    from vamtoolbox_b200.util import data as udata

    G = golden["optim"]
    s = udata.filterSinogram_t(torch.as_tensor(G["filt_sino_in"], device="cuda"), "ram-lak").cpu().numpy()
    assert np.allclose(s, G["filt_sino_ramlak"], atol=1e-10)
    t = udata.filterTargetOSMO_t(torch.as_tensor(G["target"], device="cuda"), "ram-lak").cpu().numpy()
    assert np.allclose(t, G["filt_osmo"], atol=1e-10)
    for name in ("shepp-logan", "cosine", "hamming", "hanning"):
        x = np.random.default_rng(1).uniform(size=(20, 20, 3))
        assert np.allclose(udata.filterTargetOSMO_t(torch.as_tensor(x, device="cuda"), name).cpu().numpy(),
                           udata.filterTargetOSMO(x, name), atol=1e-10), name


@pytest.mark.parametrize("engine", ["device", "host"])
@pytest.mark.parametrize("p", [2, 4])
def test_bclp_analytic_response_matches_reference(golden, engine, p):
    """BCLP with ResponseModel(type="analytical", form="gen_log_fun"): the fused device pass evaluates the
    generalised logistic and its derivative in closed form (float64 per voxel), no table."""
    from vamtoolbox_b200.optimize import optimize
    from vamtoolbox_b200.response import ResponseModel

    from vamtoolbox_b200 import geometry

    A = golden["analytic_bclp"]
    tg = geometry.TargetGeometry(target=A["target"].copy(), clip_to_circle=False)
    pg = geometry.ProjectionGeometry(A["angles"], "parallel", CUDA=True)
    rm = ResponseModel(type="analytical", form="gen_log_fun", B=12, M=0.6)
    w, lr = (1, 0.002) if p == 2 else (A["weight"], 0.02)
    sino, dose, mapped, logs = optimize(tg, pg, opts(method="BCLP", n_iter=4, p=p, q=1, eps=0.05, weight=w,
                                                     learning_rate=lr, response_model=rm, filter="ram-lak",
                                                     engine=engine), output="full")
    assert relL2(sino.array, A[f"p{p}_sino"]) < 1e-4
    assert relL2(dose.array, A[f"p{p}_dose"]) < 1e-4
    assert relL2(mapped.array, A[f"p{p}_mapped"]) < 1e-4
    assert np.allclose(logs.loss, A[f"p{p}_loss"], rtol=1e-4)


@pytest.mark.parametrize("form,kw", [("linear", {"M": 0.8, "C": 0.05}), ("identity", {})])
def test_bclp_closed_form_linear_identity_match_host_engine(form, kw):
    """The linear and identity closed forms on the device against the reference's numpy loop (host engine)."""
    from vamtoolbox_b200.optimize import optimize
    from vamtoolbox_b200.response import ResponseModel

    rng = np.random.default_rng(8)
    t = np.clip(rng.uniform(size=(24, 24, 4)), 0, 1)
    ang = np.linspace(0, 360, 18, endpoint=False)
    res = []
    for engine in ("device", "host"):
        tg, pg = geo(t, ang)
        rm = ResponseModel(type="analytical", form=form, **kw)
        res.append(optimize(tg, pg, opts(method="BCLP", n_iter=3, p=2, q=1, eps=0.05, learning_rate=0.002,
                                         response_model=rm, engine=engine), output="full"))
    assert relL2(res[0][0].array, res[1][0].array) < 1e-4
    assert relL2(res[0][2].array, res[1][2].array) < 1e-4


def test_device_metrics_match_reference(golden):
    """calcVER / calcIPDR of a CUDA tensor (fused device reductions) against the reference's values."""
    import torch

    from vamtoolbox_b200 import geometry, metrics

    G = golden["options"]
    tg = geometry.TargetGeometry(target=G["m_target"].copy())
    d = torch.as_tensor(G["m_dose"], device="cuda")
    n = np.sum(tg.gel_inds) + np.sum(tg.void_inds)
    assert abs(metrics.calcVER(tg, d) - G["m_ver"]) * n <= 1.0 + 1e-9
    assert abs(metrics.calcIPDR(tg, d) - G["m_ipdr"]) <= 1e-6 * abs(G["m_ipdr"])


def test_zslab_bclp_one_rank_equals_optimize():
    """vamtoolbox_b200.distributed.optimize_bclp_zslab on a one-rank NCCL group runs the same kernels as
    optimize() (eagerly, the loss sums passed through the all-reduce): the same sinogram, dose and loss."""
    import socket

    import torch
    import torch.distributed as dist

    from vamtoolbox_b200 import geometry, optimize as vopt
    from vamtoolbox_b200.distributed import optimize_bclp_zslab

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        rng = np.random.default_rng(4)
        t = np.zeros((48, 48, 16))
        t[14:34, 12:36, 3:13] = 1.0
        t[20:26, 20:26, :] = rng.uniform(0.3, 0.7)
        pg = geometry.ProjectionGeometry(np.linspace(0, 360, 60, endpoint=False), "parallel", CUDA=True,
                                         projector_pixel_size=0.01, absorption_coeff=2.0, container_radius=0.3)
        opts = vopt.Options(method="BCLP", n_iter=6, p=2, q=1, eps=0.1, learning_rate=1e-5)
        ref = vopt.optimize(geometry.TargetGeometry(target=t.copy()), pg, opts)
        opts2 = vopt.Options(method="BCLP", n_iter=6, p=2, q=1, eps=0.1, learning_rate=1e-5)
        got = optimize_bclp_zslab(geometry.TargetGeometry(target=t.copy()), pg, opts2)
        assert np.array_equal(ref[0].array, got[0].array)
        assert np.array_equal(ref[1].array, got[1].array)
        assert np.array_equal(np.asarray(ref[2]), np.asarray(got[2]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("method", ["OSMO", "CAL", "BCLP"])
def test_zero_dose_region_device_engine_matches_host_engine(method):
    """A target with a zero-dose region (target_geo.zero_dose, made into proj_geo.zero_dose_sino by the
    projector factory): every backprojection first sets those sinogram entries to 0 in place, as the
    reference's projectors do (Projector3DParallel.py:43-44, Projector3DParallelCUDA.py:57-58), so the
    returned sinogram is dark there, and the device engine gives the host engine's result."""
    from vamtoolbox_b200 import geometry
    from vamtoolbox_b200.optimize import optimize

    n = 40
    y, x = np.mgrid[:n, :n] - (n - 1) / 2
    body = ((x / 13.0) ** 2 + (y / 9.0) ** 2 <= 1).astype(float)
    angles = np.linspace(0, 360, 36, endpoint=False)
    out = {}
    for engine in ("device", "host"):
        tg = geometry.TargetGeometry(target=np.repeat(body[:, :, None], 4, axis=2))
        zd = np.zeros_like(tg.array)
        zd[18:22, 2:6, :] = 1.0
        tg.zero_dose = zd
        pg = geometry.ProjectionGeometry(angles, "parallel", CUDA=True)
        kw = {"OSMO": dict(n_iter=3, d_h=0.85, d_l=0.6, filter="hamming"),
              "CAL": dict(n_iter=3, learning_rate=0.4, d_h=0.5, sigmoid=0.01),
              "BCLP": dict(n_iter=3, p=2, q=1, eps=0.1, learning_rate=1e-3, filter="ram-lak")}[method]
        res = optimize(tg, pg, opts(method=method, engine=engine, **kw))
        sino = res[0].array
        assert pg.zero_dose_sino is not None and pg.zero_dose_sino.any()
        assert np.all(np.asarray(sino)[pg.zero_dose_sino] == 0), engine
        out[engine] = np.asarray(sino)
    assert relL2(out["device"], out["host"]) < 1e-4


@pytest.mark.parametrize("method", ["OSMO", "CAL"])
def test_device_engine_on_vector_geometry_matches_host_engine(method):
    """OSMO and CAL with inclined rays (the vector-geometry projector) run on the fused device engines --
    the projector's forward / backprojection into the engine's buffers, captured with the updates and
    normalisations -- and give the reference's host loop results."""
    from vamtoolbox_b200 import geometry
    from vamtoolbox_b200.optimize import optimize

    n = 32
    z, y, x = np.mgrid[:n, :n, :n] - (n - 1) / 2
    t = ((x / 10.0) ** 2 + (y / 8.0) ** 2 + (z / 12.0) ** 2 <= 1).astype(float)
    out = {}
    for engine in ("device", "host"):
        tg = geometry.TargetGeometry(target=t.copy())
        pg = geometry.ProjectionGeometry(np.linspace(0, 360, 30, endpoint=False), "parallel", CUDA=True,
                                         inclination_angle=15.0)
        kw = (dict(n_iter=4, d_h=0.85, d_l=0.6, filter="hamming") if method == "OSMO"
              else dict(n_iter=4, learning_rate=0.4, d_h=0.5, sigmoid=0.01))
        sino, recon, err = optimize(tg, pg, opts(method=method, engine=engine, **kw))
        out[engine] = (np.asarray(sino.array), np.asarray(recon.array), np.asarray(err))
    assert relL2(out["device"][0], out["host"][0]) < 1e-4
    assert relL2(out["device"][1], out["host"][1]) < 1e-4
    assert np.allclose(out["device"][2], out["host"][2], atol=2e-3, equal_nan=True)
