"""The flows of the reference's example scripts (2-D CAL / FBP with and without offset / PM / OSMO / BCLP
from an image file, a saved sinogram turned into projector frames, the .show() / .preview() calls) through
this package's public API on seeded synthetic inputs: they run end to end and give finite outputs of the
reference's shapes and types.  Parity of each optimizer is pinned elsewhere against the reference's runs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def image_file(tmp_path):
    from PIL import Image

    y, x = np.mgrid[:300, :260]
    img = (((x - 130) / 90.0) ** 2 + ((y - 150) / 70.0) ** 2 <= 1).astype(np.uint8) * 255
    img[140:160, 60:200] = 0  # a bar through the disk
    p = tmp_path / "target.png"
    Image.fromarray(img).save(p)
    return str(p)


def test_example_flows_run_end_to_end(image_file, tmp_path):
    import vamtoolbox_b200 as vam

    tg = vam.geometry.TargetGeometry(imagefilename=image_file, pixels=201)
    assert tg.array.shape[:2] == (201, 201)
    tg.show()
    angles = np.linspace(0, 360 - 360 / 180, 180)
    pg = vam.geometry.ProjectionGeometry(angles, ray_type="parallel", CUDA=True)
    for opts in (vam.optimize.Options(method="CAL", n_iter=4, d_h=0.85, d_l=0.6, filter="hamming", verbose="plot"),
                 vam.optimize.Options(method="FBP", filter="shepp-logan", verbose=None),
                 vam.optimize.Options(method="FBP", filter="shepp-logan", offset=True, verbose=None),
                 vam.optimize.Options(method="PM", filter="ram-lak", n_iter=3, d_h=0.8, d_l=0.7),
                 vam.optimize.Options(method="OSMO", filter="shepp-logan", n_iter=3, d_h=0.8, d_l=0.7)):
        sino, recon, err = vam.optimize.optimize(tg, pg, opts)
        assert sino.array.shape[:2] == (201, 180) and recon.array.shape[:2] == (201, 201)
        assert np.isfinite(sino.array).all() and np.isfinite(recon.array).all()
        if opts.method == "FBP" and getattr(opts, "offset", False):
            assert sino.array.min() >= 0.0  # offset by the magnitude of the minimum
        recon.show()
        sino.show()
    tgg = vam.geometry.TargetGeometry(imagefilename=image_file, pixels=128, binarize_image=False)
    pgg = vam.geometry.ProjectionGeometry(np.linspace(0, 180 - 180 / 90, 90), ray_type="parallel", CUDA=True)
    opts = vam.optimize.Options(method="BCLP", n_iter=5, filter="ram-lak", verbose="plot", p=2,
                                learning_rate=1e-5, response_model=vam.response.ResponseModel(B=25), eps=0.1)
    sino, recon, resp, logs = vam.optimize.optimize(tgg, pgg, opts, output="full")
    assert np.isfinite(logs.loss[:6]).all() and resp.array.shape == recon.array.shape
    logs.show()
    # a saved sinogram read back and turned into projector frames
    sino.save(str(tmp_path / "sino0"))
    loaded = vam.geometry.loadVolume(file_name=str(tmp_path / "sino0.sino"))
    assert np.array_equal(loaded.array, sino.array)
    for cfg in (vam.imagesequence.ImageConfig(image_dims=(640, 360), array_num=2, array_offset=150),
                vam.imagesequence.ImageConfig(image_dims=(640, 360), rotate_angle=45, size_scale=2)):
        seq = vam.imagesequence.ImageSeq(image_config=cfg, sinogram=loaded)
        assert len(seq.images) == 90 and seq.images[0].shape[:2] == (360, 640)
        seq.preview()
