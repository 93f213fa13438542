"""Output formats on the GPU (vam_sino_rotate / vam_sino_resize / vam_select_pair /
vam_imageseq_frames / vam_rebin_fan) against the reference's own frames and
rebinned sinograms (tests/golden/formats.npz) and the CPU oracle."""
import ctypes
import json

import numpy as np
import pytest
import torch

from oracle import formats
from vamtoolbox_b200 import _lib, geometry
from vamtoolbox_b200 import imagesequence as ims
from tests.test_formats_golden import rebin_cases, seq_cases

pytestmark = pytest.mark.gpu

# Rotation and resize sit inside scipy / OpenCV kernels whose rounding order
# is not published: the device matches them to a few ulps (checked below), so
# a frame byte may differ by one count where the value lies within those ulps
# of an integer step.  Cases without a plane transform must match exactly.
TRANSFORM_BYTE_TOL = 1e-3   # fraction of frame pixels allowed to differ by one count


def assert_frames_close(dev, ref, transformed, what):
    assert dev.shape == ref.shape and dev.dtype == np.uint8, what
    diff = dev != ref
    if not transformed:
        assert not diff.any(), (what, int(diff.sum()))
        return
    d = (dev.astype(np.int16) - ref.astype(np.int16)) % 256
    assert np.all((d[diff] == 1) | (d[diff] == 255)), what
    assert diff.mean() <= TRANSFORM_BYTE_TOL, (what, int(diff.sum()))


def test_frames_match_reference(golden):
    G = golden["formats"]
    for i, sino, kw, ref in seq_cases(G):
        seq = ims.ImageSeq(ims.ImageConfig((64, 48), **kw), sino.copy())
        dev = np.stack(seq.images)
        transformed = kw.get("rotate_angle", 0.0) != 0.0 or kw.get("size_scale", 1.0) != 1.0
        assert_frames_close(dev, ref, transformed, (i, kw))


def test_frames_from_device_tensor_and_sinogram_object(golden):
    G = golden["formats"]
    sino, kw, ref = G["seq1_sino"], json.loads(str(G["seq1_cfg"])), G["seq1_frames"]
    t = torch.from_numpy(sino).cuda()
    seq = ims.ImageSeq(ims.ImageConfig((64, 48), **kw), t, keep_device_frames=True)
    assert seq.frames_device.is_cuda and np.array_equal(seq.frames_device.cpu().numpy(), ref)
    pg = geometry.ProjectionGeometry(np.linspace(0, 360, sino.shape[1], endpoint=False))
    seq = ims.ImageSeq(ims.ImageConfig((64, 48), **kw), geometry.Sinogram(sino, pg))
    assert np.array_equal(np.stack(seq.images), ref)


def _call_rotate(x, angle, flip_r=0, flip_z=0):
    (o_r, o_z), aff = ims.rotation_plan(x.shape[0], x.shape[2], angle)
    out = torch.empty((o_r, x.shape[1], o_z), dtype=x.dtype, device="cuda")
    code = _lib.DTYPE_F64 if x.dtype == torch.float64 else _lib.DTYPE_F32
    _lib.call("vam_sino_rotate", _lib.ptr(x), code, *x.shape, flip_r, flip_z, (ctypes.c_double * 6)(*aff),
              _lib.ptr(out), o_r, o_z, _lib.stream_ptr())
    return out.cpu().numpy()


def _call_resize(x, o_r, o_z, flip_r=0, flip_z=0):
    out = torch.empty((o_r, x.shape[1], o_z), dtype=torch.float64, device="cuda")
    code = _lib.DTYPE_F64 if x.dtype == torch.float64 else _lib.DTYPE_F32
    _lib.call("vam_sino_resize", _lib.ptr(x), code, *x.shape, flip_r, flip_z, _lib.ptr(out), o_r, o_z,
              _lib.stream_ptr())
    return out.cpu().numpy()


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("angle", [30.0, -12.5, 90.0, 123.4, 7.0])
def test_rotate_matches_oracle(dtype, angle):
    rng = np.random.default_rng(3)
    x = rng.random((37, 5, 29)).astype(dtype)
    dev = _call_rotate(torch.from_numpy(x).cuda(), angle)
    ref = formats.rotate_planes(x, angle)
    assert dev.dtype == ref.dtype and np.array_equal(dev, ref)
    # flips folded into the kernel equal a flipped input
    dev_f = _call_rotate(torch.from_numpy(x).cuda(), angle, 1, 1)
    assert np.array_equal(dev_f, formats.rotate_planes(np.ascontiguousarray(x[::-1, :, ::-1]), angle))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("scale", [1.5, 0.7, 2.0, 0.5, 1.25])
def test_resize_matches_oracle(dtype, scale):
    rng = np.random.default_rng(4)
    x = rng.random((40, 6, 26)).astype(dtype)
    o_r, o_z = int(40 * scale), int(26 * scale)
    dev = _call_resize(torch.from_numpy(x).cuda(), o_r, o_z)
    ref = formats.resize_planes(x, scale)
    assert np.array_equal(dev, ref)
    dev_f = _call_resize(torch.from_numpy(x).cuda(), o_r, o_z, 1, 0)
    assert np.array_equal(dev_f, formats.resize_planes(np.ascontiguousarray(x[::-1]), scale))


def _select(x, k0, k1):
    t = torch.as_tensor(x).cuda()
    code = _lib.DTYPE_F64 if t.dtype == torch.float64 else _lib.DTYPE_F32
    out = torch.empty(2, dtype=t.dtype, device="cuda")
    nb = _lib.load().vam_select_workspace_bytes()
    work = torch.empty(nb, dtype=torch.uint8, device="cuda")
    _lib.call("vam_select_pair", _lib.ptr(t), code, t.numel(), k0, k1, _lib.ptr(out), _lib.ptr(work), nb,
              _lib.stream_ptr())
    return out.cpu().numpy()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_select_pair_matches_sort(dtype):
    rng = np.random.default_rng(9)
    cases = [
        rng.standard_normal(100_003),
        np.concatenate([np.zeros(50_000), rng.random(1000), np.full(20, -3.5)]),   # long runs of equal keys
        np.full(4097, 2.25),
        np.array([7.0]),
        np.array([-0.0, 0.0, -1.0, 1.0, np.inf, -np.inf, 5e-310, -5e-310]),
        rng.integers(-3, 4, size=33_333).astype(np.float64),
        rng.random(3_000_000) * 1e6,
    ]
    for x in cases:
        x = x.astype(dtype)
        n = x.size
        s = np.sort(x)
        for k0 in sorted({0, n // 3, n // 2, max(n - 2, 0), n - 1}):
            for k1 in {k0, min(k0 + 1, n - 1)}:
                got = _select(x, k0, k1)
                assert got[0] == s[k0] and got[1] == s[k1], (n, k0, k1, got, s[k0], s[k1])


def test_select_pair_nan_gives_nan():
    x = np.arange(1000, dtype=np.float64)
    x[17] = np.nan
    got = _select(x, 10, 11)
    assert np.isnan(got).all()


def test_select_pair_argument_errors():
    lib = _lib.load()
    assert lib.vam_select_pair(None, 0, 10, 0, 0, None, None, 0, None) == _lib.VAM_ERR_ARG
    t = torch.zeros(10, device="cuda")
    out = torch.empty(2, device="cuda")
    w = torch.empty(lib.vam_select_workspace_bytes(), dtype=torch.uint8, device="cuda")
    nb = w.numel()
    assert lib.vam_select_pair(_lib.ptr(t), 0, 10, 3, 5, _lib.ptr(out), _lib.ptr(w), nb, None) == _lib.VAM_ERR_ARG
    assert lib.vam_select_pair(_lib.ptr(t), 0, 10, 9, 10, _lib.ptr(out), _lib.ptr(w), nb, None) == _lib.VAM_ERR_ARG
    assert lib.vam_select_pair(_lib.ptr(t), 0, 0, 0, 0, _lib.ptr(out), _lib.ptr(w), nb, None) == _lib.VAM_ERR_SHAPE


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_full_screen_frames_match_oracle(dtype):
    """A 1920 x 1080 frame sequence at the bench's configuration (no plane transform): exact."""
    rng = np.random.default_rng(21)
    sino = (rng.random((256, 48, 256)) ** 3 * 40.0).astype(dtype)
    sino[:20] = 0
    kw = dict(normalization_percentile=99.5, intensity_scale=0.9, invert_u=True, v_offset=-40, u_offset=100)
    dev = np.stack(ims.ImageSeq(ims.ImageConfig((1920, 1080), **kw), sino).images)
    ref = formats.image_frames(sino, formats.config(1920, 1080, **kw))
    assert_frames_close(dev, ref, False, kw)


def test_frames_bit_depths_and_wraparound():
    """Values past 255 in 10/16/32-bit sequences keep their low byte, as the uint8 frame store does."""
    rng = np.random.default_rng(5)
    sino = rng.random((32, 9, 28)) * 5000.0
    sino[0, :, 0] = np.nan
    sino[1, :, 1] = -7.25
    for kw in [dict(bit_depth=10), dict(bit_depth=16, intensity_scale=17.0), dict(bit_depth=32, intensity_scale=1e6),
               dict(bit_depth=0), dict(bit_depth=8, normalization_percentile=0)]:
        dev = np.stack(ims.ImageSeq(ims.ImageConfig((64, 48), **kw), sino).images)
        with np.errstate(all="ignore"):
            ref = formats.image_frames(sino, formats.config(64, 48, **kw))
        assert np.array_equal(dev, ref), kw


def test_frames_reject_unsupported_input():
    with pytest.raises(TypeError):
        ims.ImageSeq(ims.ImageConfig((64, 48)), np.zeros((4, 3, 4), dtype=np.int32))
    with pytest.raises(ctypes.ArgumentError):
        ims.ImageSeq(ims.ImageConfig((64, 48)), [1, 2, 3])
    with pytest.raises(ValueError, match="Bit depth higher than 32-bit"):
        ims.ImageSeq(ims.ImageConfig((64, 48), bit_depth=40), np.zeros((4, 3, 4)))


def test_rebin_matches_reference_bitwise(golden):
    G = golden["formats"]
    for i, sino, angles, (vw, scr, n_write, throw), ref in rebin_cases(G):
        pg = geometry.ProjectionGeometry(angles)
        s = geometry.Sinogram(sino.copy(), pg)
        out = geometry.rebinFanBeam(s, vw, scr, n_write, throw)
        assert isinstance(out.array, np.ndarray) and out.array.dtype == ref.dtype
        assert np.array_equal(out.array, ref), i
        # the input Sinogram's array is replaced by its padded copy, as in the reference
        assert s.array.shape[0] == vw
        # a device tensor stays on the device
        s_t = geometry.Sinogram(torch.from_numpy(sino.copy()).cuda(), pg)
        out_t = geometry.rebinFanBeam(s_t, vw, scr, n_write, throw)
        assert out_t.array.is_cuda and np.array_equal(out_t.array.cpu().numpy(), ref), i
        assert tuple(s_t.array.shape)[0] == vw


def test_rebin_rejects_too_narrow_vial():
    pg = geometry.ProjectionGeometry(np.linspace(0, 360, 10, endpoint=False))
    with pytest.raises(ValueError):
        geometry.rebinFanBeam(geometry.Sinogram(np.zeros((30, 10, 2)), pg), 20, (1920, 1080), 1.5, 1.7)


@pytest.mark.parametrize("shape,screen,kw", [
    ((37, 5, 23), (68, 52), dict(normalization_percentile=95.0)),                 # odd window, n_u % 16 != 0
    ((24, 4, 20), (64, 100), dict(array_num=4, array_offset=12, invert_v=True)),  # overlapping copies
    ((24, 4, 20), (64, 100), dict(array_num=3, array_offset=30, v_offset=4)),     # gaps between copies
    ((30, 3, 18), (96, 64), dict(rotate_angle=20.0, size_scale=1.3, invert_u=True)),
    ((16, 2, 16), (64, 48), dict(array_num=0)),                                   # nothing inserted
])
def test_device_frames_and_images_match_oracle(shape, screen, kw):
    rng = np.random.default_rng(17)
    sino = rng.random(shape) * 300.0
    cfg = ims.ImageConfig(screen, **kw)
    seq = ims.ImageSeq(cfg, sino, keep_device_frames=True)
    full = seq.frames_device.cpu().numpy()
    assert np.array_equal(full, np.stack(seq.images))
    ref = formats.image_frames(sino, formats.config(*screen, **kw))
    transformed = "rotate_angle" in kw or "size_scale" in kw
    assert_frames_close(full, ref, transformed, kw)
