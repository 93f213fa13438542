"""The reference's small util modules: thresholding.threshold, timing.timing, matlab.saveMatData
(vamtoolbox/util/thresholding.py, timing.py, matlab.py) on the host, and build_sparse_matrix.buildMatrix
(vamtoolbox/util/build_sparse_matrix.py) on the device: its rows are the projector's backprojections of
unit sinograms, so P^T b equals the backprojection of b."""
import numpy as np
import pytest
import scipy.io


def test_threshold_timing_and_matlab(tmp_path, capsys):
    from vamtoolbox_b200 import geometry
    from vamtoolbox_b200.util import matlab, thresholding, timing

    x = np.array([[0.2, 0.5], [0.7, 0.49]])
    t = thresholding.threshold(x, 0.5)
    assert t.dtype == np.bool_ and t.tolist() == [[False, True], [True, False]]

    @timing.timing
    def twice(v):
        return 2 * v

    assert twice(3) == 6 and "twice function took" in capsys.readouterr().out
    tg = geometry.TargetGeometry(target=x.copy())
    sino = geometry.Sinogram(np.arange(6.0).reshape(3, 2), geometry.ProjectionGeometry(np.array([0.0, 90.0]), "parallel"))
    f = tmp_path / "out.mat"
    matlab.saveMatData(str(f), target_geo=tg, sinogram=sino)
    d = scipy.io.loadmat(str(f))
    assert np.array_equal(d["target"], tg.array)
    assert np.array_equal(d["opt_proj"], sino.array)
    with pytest.raises(Exception):
        matlab.saveMatData(str(f), sinogram=np.zeros(3))


@pytest.mark.gpu
def test_build_matrix_rows_are_unit_backprojections():
    from vamtoolbox_b200 import geometry
    from vamtoolbox_b200.projectorconstructor import projectorconstructor
    from vamtoolbox_b200.util.build_sparse_matrix import buildMatrix

    rng = np.random.default_rng(5)
    tg = geometry.TargetGeometry(target=rng.uniform(0, 1, (12, 12)))
    pg = geometry.ProjectionGeometry(np.linspace(0, 180, 7, endpoint=False), "parallel", CUDA=True)
    P = buildMatrix(tg, pg)
    A = projectorconstructor(tg, pg)
    b = rng.uniform(0, 1, np.asarray(A.forward(np.zeros_like(tg.array))).shape)
    want = np.asarray(A.backward(b.copy())).ravel()
    got = P.T @ b.ravel()
    assert np.linalg.norm(got - want) <= 1e-5 * np.linalg.norm(want)
    assert P.format == "csr" and P.shape == (b.size, tg.array.size)


def test_package_namespace_and_resources(tmp_path, monkeypatch):
    """The reference's examples use vam.optimize / vam.response / vam.imagesequence / vam.resources right
    after `import vamtoolbox as vam`; resources.load resolves the reference's names in a resource folder."""
    from argparse import ArgumentError

    import vamtoolbox_b200 as vam

    for name in ("optimize", "response", "metrics", "imagesequence", "resources", "projector", "optimizer",
                 "projectorconstructor", "geometry", "medium", "util"):
        assert hasattr(vam, name), name
    assert callable(vam.optimize.optimize) and callable(vam.optimize.Options)
    monkeypatch.setenv("VAMTOOLBOX_RESOURCES", str(tmp_path))
    assert vam.resources.load("Flower.png") == str(tmp_path / "flower.png")
    with pytest.raises(ArgumentError):
        vam.resources.load("teapot.stl")


def test_show_is_headless(caplog):
    """The reference's examples end with .show() on targets, sinograms, reconstructions and loss logs; here
    those calls log that nothing is drawn and return, so the scripts finish on a headless machine."""
    from vamtoolbox_b200 import geometry
    from vamtoolbox_b200.optimize import Options
    from vamtoolbox_b200.optimizer.BCLP import LogPerf

    from vamtoolbox_b200 import medium
    from vamtoolbox_b200.response import ResponseModel

    tg = geometry.TargetGeometry(target=np.ones((8, 8)))
    cv = tg.constructCoordVec()
    with caplog.at_level("WARNING"):
        assert tg.show() is None
        assert LogPerf(Options(method="BCLP", n_iter=2)).show() is None
        im = medium.IndexModel(cv, type="analytical", form="homogeneous")
        am = medium.AttenuationModel(cv, type="analytical", form="homogeneous_cylinder", R=1, alpha_internal=0.2)
        assert im.plotIndex(block=False) is None and am.plotAlpha(block=True) is None
        assert ResponseModel(form="gen_log_fun", B=10).plotMap(None, None, label="B=10") is None
    assert caplog.text.count("no display") >= 5
