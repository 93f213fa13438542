"""Dose metrics (vamtoolbox_b200.metrics, host numpy path) against the
reference's own calcVER / calcIPDR / calcPW / calcCV on a seeded target and
dose (tests/golden/options.npz).  Exact up to float64 summation order."""
import numpy as np

from tests.conftest import relL2  # noqa: F401  (shared helpers live there)


def test_metrics_match_reference(golden):
    from vamtoolbox_b200 import geometry, metrics

    G = golden["options"]
    tg = geometry.TargetGeometry(target=G["m_target"].copy())
    d = G["m_dose"]
    assert metrics.calcVER(tg, d) == G["m_ver"]
    assert metrics.calcIPDR(tg, d) == G["m_ipdr"]
    assert metrics.calcPW(tg, d) == G["m_pw"]
    assert np.isclose(metrics.calcCV(tg, d), G["m_cv"], rtol=1e-12, atol=0)


def test_layerwise_metrics_are_per_slice_whole_volume_values(golden):
    """The layerwise forms (which raise IndexError in the reference) reduce each slice on its own: for
    a one-slice target they equal the whole-volume values."""
    from vamtoolbox_b200 import geometry, metrics

    G = golden["options"]
    t, d = G["m_target"][:, :, 1:2].copy(), G["m_dose"][:, :, 1:2]
    tg = geometry.TargetGeometry(target=t)
    for fn in (metrics.calcVER, metrics.calcIPDR, metrics.calcPW):
        assert fn(tg, d, layerwise=True)[0] == fn(tg, d)
