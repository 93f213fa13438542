"""Batched calls (vam_batch_*): many plans of uneven size in one persistent launch.

Every call in a batch runs the body its plan's own entry point runs, so batch
outputs must equal the single-call outputs bit for bit (the kernels are
deterministic gathers).  Covers 2-D slices, 3-D volumes on the generic and the
fast (4 and 8 slices per lane) paths, mask / ray absorption, occlusion, all
three ops, resubmission, graph capture and the multi-target BCLP engine."""
import numpy as np
import pytest
import torch

from vamtoolbox_b200 import _lib
from vamtoolbox_b200.batch import ProjectionBatch
from vamtoolbox_b200.projector.Projector3DParallel import ParallelPlan

pytestmark = pytest.mark.gpu


def make_plans(seed=0):
    rng = np.random.default_rng(seed)
    specs = [((40, 40, 1), 36, "mask"), ((24, 24, 64), 30, None), ((20, 20, 96), 18, "ray"),
             ((16, 16, 256), 24, "mask"), ((33, 33, 128), 20, None), ((18, 18, 8), 12, "occ"),
             ((31, 31, 1), 45, "ray")]
    out = []
    for shape, na, mode in specs:
        ang = np.linspace(0, 360, na, endpoint=False) + (0.0 if na % 2 == 0 else 1.3)
        p = ParallelPlan(shape[0], shape[1], shape[2], ang)
        if mode == "mask":
            p.set_absorption("mask", mask=rng.uniform(0.3, 1.0, shape[:2]))
        elif mode == "ray":
            p.set_absorption("ray", alpha_per_px=0.03, radius_px=shape[0] / 2 - 1.5)
        elif mode == "occ":
            ins = np.zeros(shape)
            ins[7:10, 6:9, :] = 1.0
            p.set_occlusion(ins)
        x = torch.as_tensor(rng.uniform(0, 1, shape), dtype=torch.float32, device="cuda")
        b = torch.as_tensor(rng.uniform(0, 1, p.shape_sino), dtype=torch.float32, device="cuda")
        out.append((p, x, b))
    return out


def work_list(plans):
    work, outs = [], []
    for p, x, b in plans:
        ob, ox, oa = torch.full_like(b, np.nan), torch.full_like(x, np.nan), torch.full_like(x, np.nan)
        work += [(p, "forward", x, ob), (p, "backward_ref", b, ox), (p, "adjoint", b, oa)]
        outs.append((ob, ox, oa))
    return work, outs


def single(plans):
    return [(p.forward(x), p.backward_ref(b), p.adjoint(b)) for p, x, b in plans]


def test_batch_equals_single_calls_bitwise():
    plans = make_plans()
    ref = single(plans)
    batch = ProjectionBatch()
    work, outs = work_list(plans)
    batch.submit(work)
    torch.cuda.synchronize()
    for (rf, rb, ra), (of, ob, oa) in zip(ref, outs):
        assert torch.equal(rf, of)
        assert torch.equal(rb, ob)
        assert torch.equal(ra, oa)
    info = batch.info()
    assert info["ctas"] > 0 and info["virtual_blocks"] >= info["ctas"]


def test_batch_resubmit_and_new_list():
    plans = make_plans(1)
    ref = single(plans)
    batch = ProjectionBatch()
    work, outs = work_list(plans)
    batch.submit(work)
    for o in outs:
        for t in o:
            t.fill_(np.nan)
    batch.submit(work)  # same list: launch only
    torch.cuda.synchronize()
    for r, o in zip(ref, outs):
        assert all(torch.equal(a, c) for a, c in zip(r, o))
    # a shorter, different list on the same batch
    work2, outs2 = work_list(plans[:3])
    batch.submit(work2)
    torch.cuda.synchronize()
    for r, o in zip(ref[:3], outs2):
        assert all(torch.equal(a, c) for a, c in zip(r, o))


def test_batch_graph_capture():
    """A never-submitted list is captured directly (descriptions travel in the launch parameters)."""
    plans = make_plans(2)
    ref = single(plans)
    batch = ProjectionBatch()
    work, outs = work_list(plans)
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=s):
        batch.submit(work)
    for _ in range(2):
        for o in outs:
            for t in o:
                t.fill_(np.nan)
        g.replay()
        torch.cuda.synchronize()
        for r, o in zip(ref, outs):
            assert all(torch.equal(a, c) for a, c in zip(r, o))
    del g


def test_batch_long_list_spans_launches():
    """More calls than one launch carries (48): consecutive persistent launches, same results."""
    plans = make_plans(4)
    ref = single(plans)
    batch = ProjectionBatch()
    work, outs = [], []
    for rep in range(8):  # 7 plans x (bwd + adj) x 8 = 112 calls, forwards once per plan
        for p, x, b in plans:
            ox, oa = torch.full_like(x, np.nan), torch.full_like(x, np.nan)
            work += [(p, "backward_ref", b, ox), (p, "adjoint", b, oa)]
            outs.append((ox, oa))
    batch.submit(work)
    torch.cuda.synchronize()
    for k, (ox, oa) in enumerate(outs):
        _, rb, ra = ref[k % len(plans)]
        assert torch.equal(rb, ox) and torch.equal(ra, oa)


def test_batch_large_calls_bitwise():
    """Calls large enough for the 2-D tile bodies (forward from 192 px, backprojection from 320 px), the
    generic 3-D bodies at nZ = 160 and the fast ones, with more blocks than resident CTAs, so the CTAs
    fetch their next ticket while a block runs and switch to one ticket at a time near the end."""
    rng = np.random.default_rng(7)
    plans = []
    for shape, na, mode in [((256, 256, 1), 90, "mask"), ((352, 352, 1), 60, None), ((258, 258, 1), 45, None),
                            ((363, 363, 1), 36, "mask"), ((228, 228, 1), 40, "plain"),
                            ((96, 96, 160), 40, "mask"), ((64, 64, 96), 120, None),
                            ((64, 64, 256), 72, "table"), ((49, 49, 128), 60, "table")]:
        p = ParallelPlan(shape[0], shape[1], shape[2], np.linspace(0, 360, na, endpoint=False))
        if mode == "mask":
            p.set_absorption("mask", mask=rng.uniform(0.3, 1.0, shape[:2]))
        elif mode == "plain":  # the 2-D forward with plain-load staging runs in the all-bodies instance
            p.set_tuning({"forward_tma": 0})
        elif mode == "table":  # block-table backprojection (eight and four slices per lane)
            assert p.prepare_backward()
        x = torch.as_tensor(rng.uniform(0, 1, shape), dtype=torch.float32, device="cuda")
        b = torch.as_tensor(rng.uniform(0, 1, p.shape_sino), dtype=torch.float32, device="cuda")
        plans.append((p, x, b))
    ref = [(p.forward(x), p.backward_ref(b)) for p, x, b in plans]
    batch = ProjectionBatch()
    work, outs = [], []
    for p, x, b in plans:
        ob, ox = torch.full_like(b, np.nan), torch.full_like(x, np.nan)
        work += [(p, "forward", x, ob), (p, "backward_ref", b, ox)]
        outs.append((ob, ox))
    for _ in range(2):  # a resubmission reuses the prepared list
        batch.submit(work)
        torch.cuda.synchronize()
        for (rf, rb), (of, ob) in zip(ref, outs):
            assert torch.equal(rf, of)
            assert torch.equal(rb, ob)
        for o in outs:
            for t in o:
                t.fill_(np.nan)
    assert batch.info()["virtual_blocks"] > 2 * 148 * 6


def test_batch_rejects_bad_work():
    plans = make_plans(3)
    batch = ProjectionBatch()
    p, x, b = plans[1]
    with pytest.raises(ValueError):
        batch.submit([(p, "sideways", x, b)])
    with pytest.raises(ValueError):
        batch.submit([(p, "forward", b, x)])  # shapes swapped
    h = _lib.load()
    assert h.vam_batch_submit(batch._h, None, 0, None) == _lib.VAM_ERR_ARG
    # two forwards of one plan that both stage their input (a 2-D slice whose rows are not a multiple of
    # 16 bytes) would share the plan's padded image: refused, nothing launched
    q = ParallelPlan(198, 198, 1, np.linspace(0, 180, 30, endpoint=False))
    x1, x2 = torch.rand(198, 198, 1, device="cuda"), torch.rand(198, 198, 1, device="cuda")
    o1, o2 = torch.zeros(q.shape_sino, device="cuda"), torch.zeros(q.shape_sino, device="cuda")
    with pytest.raises(_lib.VamError) as e:
        batch.submit([(q, "forward", x1, o1), (q, "forward", x2, o2)])
    assert e.value.code == _lib.VAM_ERR_ARG and "same scratch" in e.value.message
    batch.submit([(q, "forward", x1, o1)])
    torch.cuda.synchronize()
    assert torch.equal(o1, q.forward(x1))


@pytest.mark.parametrize("schedule", ["persistent", "streams", "phased", "auto"])
def test_multi_target_bclp_matches_one_at_a_time(schedule):
    from vamtoolbox_b200 import geometry
    from vamtoolbox_b200.optimize import Options
    from vamtoolbox_b200.optimizer.BCLP import BCLPNorm
    from vamtoolbox_b200.optimizer.multi import MultiTargetBCLP
    from vamtoolbox_b200.synthetic import ellipses_2d, ellipsoids_3d

    probs = []
    for k, (n, nz, na, a) in enumerate([(48, 1, 60, 2.0), (32, 64, 36, 0.0), (24, 128, 24, 4.0)]):
        t = ellipses_2d(n, seed=k, radius=0.45 * n) if nz == 1 else ellipsoids_3d(n, nz, seed=k, radius=0.45 * n)
        tg = geometry.TargetGeometry(target=t)
        pg = geometry.ProjectionGeometry(np.linspace(0, 360, na, endpoint=False), "parallel", CUDA=True,
                                         projector_pixel_size=0.01, absorption_coeff=a if a else None,
                                         container_radius=n * 0.005)
        opts = Options(method="BCLP", n_iter=6, p=2, q=1, eps=0.1, learning_rate=0.01)
        probs.append((tg, pg, opts))
    multi = MultiTargetBCLP(probs, schedule=schedule).run()
    for (tg, pg, opts), (g, dose, loss) in zip(probs, multi):
        s = BCLPNorm(tg, pg, opts)
        g1 = s.checkSinogramShape(s.gradientDescent(), "cylindrical")
        assert np.array_equal(g, g1)
        assert np.array_equal(dose, s.dose)
        assert np.allclose(np.asarray(loss), np.asarray(s.logs.loss), rtol=0, atol=0, equal_nan=True)
