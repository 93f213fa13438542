"""util.data's target filters and contrast stretch against the reference's own outputs
(tests/golden/datafilters.npz, made by tests/golden/make_golden.py from vamtoolbox/util/data.py):
filterTargetBCLP (util/data.py:116-196), filterTarget (:199-300) for every filter name on a 2-D and a
3-D input, and histogramEqualization (:471-492).  Host numpy code, no GPU."""
import numpy as np
import pytest

from vamtoolbox_b200.util import data as D

NAMES = ("ram-lak", "shepp-logan", "cosine", "hamming", "hanning")


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("tag", ["x2", "x3"])
def test_target_filters_match_reference(golden, name, tag):
    G = golden["datafilters"]
    x = G[tag]
    np.testing.assert_allclose(D.filterTargetBCLP(x.copy(), name), G[f"bclp_{name}_{tag}"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(D.filterTarget(x.copy(), name), G[f"target_{name}_{tag}"], rtol=1e-12, atol=1e-12)


def test_target_filter_edge_cases(golden):
    x = golden["datafilters"]["x2"]
    assert D.filterTargetBCLP(x, None) is x
    # the reference checks the name list (which holds None, not "none") before its "none" branch
    for bad in ("none", "box"):
        with pytest.raises(ValueError):
            D.filterTargetBCLP(x, bad)
    with pytest.raises(AssertionError):
        D.filterTarget(np.zeros((8, 9)), "ram-lak")


def test_histogram_equalization_matches_reference(golden):
    G = golden["datafilters"]
    np.testing.assert_array_equal(D.histogramEqualization(G["h"].copy(), 8), G["histeq"])
