"""Fused optimizer kernels (csrc/optim.cu) against numpy restatements of the
reference's iteration bodies."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def ws():
    from vamtoolbox_b200.fused import Workspace

    return Workspace("cuda")


@pytest.mark.parametrize("n", [1, 7, 1000, 3_000_001])
def test_reductions(n):
    from vamtoolbox_b200 import _lib

    w = ws()
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n).astype(np.float32)
    t = torch.as_tensor(x, device="cuda")
    out = w.scalar()
    for op, ref in ((_lib.RED_MAX, x.max()), (_lib.RED_MIN, x.min()), (_lib.RED_SUM, x.astype(np.float64).sum())):
        w.reduce(t, op, out)
        assert np.isclose(float(out.item()), ref, rtol=1e-6, atol=1e-6)


def test_max_propagates_nan():
    w = ws()
    t = torch.ones(100, device="cuda")
    t[37] = float("nan")
    out = w.scalar()
    w.max(t, out)
    assert np.isnan(float(out.item()))


def test_ver_matches_numpy():
    from types import SimpleNamespace

    from vamtoolbox_b200 import metrics

    rng = np.random.default_rng(0)
    x = rng.uniform(size=(40, 40, 6)).astype(np.float32)
    gel = rng.uniform(size=x.shape) > 0.6
    void = ~gel & (rng.uniform(size=x.shape) > 0.2)
    tg = SimpleNamespace(gel_inds=gel, void_inds=void)
    w = ws()
    out = w.scalar()
    w.ver(torch.as_tensor(x, device="cuda"), torch.as_tensor(metrics.region_mask(tg), device="cuda"), out)
    assert np.isclose(float(out.item()), metrics.calcVER(tg, x), rtol=0, atol=1e-7)


@pytest.mark.parametrize("p", [2.0, 4.0, 1.5])
def test_bclp_dose_pass_matches_reference_body(p):
    from vamtoolbox_b200.fused import bclp_params
    from vamtoolbox_b200.response import ResponseModel

    rng = np.random.default_rng(int(p * 10))
    dose = rng.uniform(-0.1, 1.2, (30, 30, 5))
    target = np.round(rng.uniform(size=dose.shape) * 2) / 2
    weight = np.where(target > 0, 1.0, 0.5)
    rm = ResponseModel(B=12, M=0.6)
    keep = []
    wt = torch.as_tensor(weight.astype(np.float32), device="cuda")
    prm = bclp_params(rm, 0.05, wt, p, torch.device("cuda"), keep)
    w = ws()
    d, t = (torch.as_tensor(a.astype(np.float32), device="cuda") for a in (dose, target))
    mapped, operand, stats = torch.empty_like(d), torch.empty_like(d), w.scalar(9)
    w.bclp_dose_pass(d, t, prm, mapped, operand, stats)
    m_ref, op_ref, st_ref = O.bclp_dose_pass(dose.astype(np.float32).astype(np.float64), target, rm.interp_f_0,
                                             rm.interp_map_0, rm.interp_dmapdf_0, 0.05, weight, p)
    assert np.allclose(mapped.cpu().numpy(), m_ref, atol=2e-6)
    assert np.allclose(operand.cpu().numpy(), op_ref, atol=1e-4 * np.abs(op_ref).max())
    st = stats.cpu().numpy()
    assert np.allclose(st[[1, 2]], st_ref[[1, 2]], atol=2)  # voxel counts
    assert np.allclose(st[[0, 3, 4, 5, 6, 7, 8]], st_ref[[0, 3, 4, 5, 6, 7, 8]], rtol=2e-4)


def test_bclp_update_prefactor_and_zero_loss():
    w = ws()
    g = torch.full((1000,), 0.5, device="cuda")
    grad = torch.full((1000,), 2.0, device="cuda")
    stats = w.scalar(9)
    stats[0] = 4.0  # sum -> loss = 4^(q/p) = 2 with p=2, q=1 -> pref = q L^((q-p)/q) = 0.5
    w.bclp_update(g, grad, 0.1, 2.0, 1.0, 0.0, None, stats)
    assert torch.allclose(g, torch.full_like(g, 0.5 - 0.1 * 0.5 * 2.0))
    stats[0] = 0.0  # loss == 0: no prefactor (BCLP.py:370-375)
    g.fill_(0.5)
    w.bclp_update(g, grad, 0.1, 2.0, 1.0, 0.0, 0.45, stats)
    assert torch.allclose(g, torch.full_like(g, 0.3))
    g.fill_(0.5)
    w.bclp_update(g, grad, 1.0, 2.0, 1.0, 0.0, None, stats)
    assert float(g.min()) == 0.0


def test_append_counts_rows_and_caps():
    w = ws()
    log = torch.full((3, 2), -1.0, device="cuda")
    ctr = torch.zeros(1, dtype=torch.int32, device="cuda")
    for v in range(5):
        w.append(torch.tensor([v, v + 10.0], device="cuda"), log, ctr)
    assert int(ctr.item()) == 5
    assert log.cpu().tolist() == [[0, 10], [1, 11], [2, 12]]
