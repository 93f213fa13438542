"""Output formats on the CPU: the oracle against the reference's own frames and
rebinned sinograms (tests/golden/formats.npz), and the host-side pieces of the
device pipeline (placement tables, percentile ranks and blend, rotation plan)."""
import json

import numpy as np
import pytest
from scipy import ndimage

from oracle import formats
from vamtoolbox_b200 import imagesequence as ims


def seq_cases(G):
    i = 0
    while f"seq{i}_sino" in G.files:
        yield i, G[f"seq{i}_sino"], json.loads(str(G[f"seq{i}_cfg"])), G[f"seq{i}_frames"]
        i += 1


def rebin_cases(G):
    i = 0
    while f"rebin{i}_sino" in G.files:
        vw, nu, nv, n_write, throw = G[f"rebin{i}_args"]
        yield i, G[f"rebin{i}_sino"], G[f"rebin{i}_angles"], (int(vw), (int(nu), int(nv)), n_write, throw), \
            G[f"rebin{i}_out"]
        i += 1


def test_oracle_frames_match_reference(golden):
    G = golden["formats"]
    n = 0
    for i, sino, kw, ref in seq_cases(G):
        mine = formats.image_frames(sino, formats.config(64, 48, **kw))
        assert mine.dtype == np.uint8 and mine.shape == ref.shape, i
        assert np.array_equal(mine, ref), (i, kw, int((mine != ref).sum()))
        n += 1
    assert n >= 15


def test_oracle_rebin_matches_reference_bitwise(golden):
    G = golden["formats"]
    n = 0
    for i, sino, angles, (vw, scr, n_write, throw), ref in rebin_cases(G):
        mine = formats.rebin_fan(sino, angles, vw, scr, n_write, throw)
        assert mine.dtype == ref.dtype and np.array_equal(mine, ref), i
        n += 1
    assert n >= 4


@pytest.mark.parametrize("shape,angle", [((24, 20), 30.0), ((37, 23), -12.5), ((19, 30), 90.0), ((64, 48), 123.4)])
def test_rotation_plan_is_scipys(shape, angle):
    (o_r, o_z), aff = ims.rotation_plan(shape[0], shape[1], angle)
    x = np.zeros((shape[0], 2, shape[1]))
    assert ndimage.rotate(x, angle, axes=(0, 2), reshape=True, order=1).shape == (o_r, 2, o_z)
    # the oracle's rotation (pinned against the reference above) agrees with scipy to a few ulps
    rng = np.random.default_rng(0)
    x = rng.random((shape[0], 3, shape[1]))
    ref = ndimage.rotate(x, angle, axes=(0, 2), reshape=True, order=1)
    assert np.max(np.abs(formats.rotate_planes(x, angle) - ref)) < 1e-14


def _np_percentile_via_pair(a, p):
    s = np.sort(a.ravel())
    k0, k1, g = ims.percentile_ranks(a.size, p, a.dtype)
    return ims.blend(s[k0], s[k1], g)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_percentile_ranks_and_blend_reproduce_numpy(dtype):
    rng = np.random.default_rng(11)
    for _ in range(300):
        n = int(rng.integers(1, 4000))
        a = (rng.random(n) * rng.choice([1.0, 1e3, 1e-3])).astype(dtype)
        p = rng.choice([0, 50, 99, 99.5, 99.9, 100, 12.5, float(rng.random() * 100)])
        p = rng.choice([float(p), np.float64(p), np.float32(p), int(round(p))])
        ref = np.percentile(a, p)
        mine = _np_percentile_via_pair(a, p)
        assert mine == ref and np.asarray(mine).dtype == np.asarray(ref).dtype, (n, p, type(p))


def test_percentile_out_of_range_raises():
    with pytest.raises(ValueError, match="Percentiles must be in the range"):
        ims.percentile_ranks(10, 101.0, np.dtype(np.float64))


def test_placement_tables_reproduce_insertion():
    rng = np.random.default_rng(2)
    for kw in [dict(), dict(u_offset=5, v_offset=-3), dict(array_num=3, array_offset=9, v_offset=1),
               dict(array_num=4, array_offset=7), dict(array_num=0), dict(invert_u=True, invert_v=True)]:
        cfg = formats.config(64, 48, **kw)
        q = rng.integers(0, 255, size=(24, 3, 20)).astype(np.uint8)
        frames = np.zeros((3, 48, 64), np.uint8)
        oracle_frames = formats.image_frames(q.astype(np.float64), cfg)
        col, row = ims.placement_tables(ims.ImageConfig((64, 48), **kw), 24, 20, 24, 20, kw.get("invert_u", False),
                                        kw.get("invert_v", False))
        for a in range(3):
            for v in range(48):
                for u in range(64):
                    if col[u] >= 0 and row[v] >= 0:
                        frames[a, v, u] = q[col[u], a, row[v]]
        assert np.array_equal(frames, oracle_frames), kw


def test_placement_errors_mirror_reference():
    with pytest.raises(Exception, match="too large in the u-dimension"):
        ims.placement_tables(ims.ImageConfig((16, 48)), 24, 20, 24, 20)
    with pytest.raises(Exception, match="too large in the v-dimension"):
        ims.placement_tables(ims.ImageConfig((64, 48), v_offset=20), 24, 20, 24, 20)
    with pytest.raises(ValueError, match="could not broadcast"):
        ims.placement_tables(ims.ImageConfig((8, 48)), 9, 20, 9, 20)
    with pytest.raises(Exception, match="divisible by 4"):
        ims.ImageConfig((62, 48))


def test_copy_offsets_sequences():
    cfg = ims.ImageConfig((64, 48), array_num=4, array_offset=10, v_offset=2)
    assert ims.copy_offsets(cfg) == [7, -3, 12, -8]
    cfg = ims.ImageConfig((64, 48), array_num=3, array_offset=10, v_offset=2)
    assert ims.copy_offsets(cfg) == [2, 12, -8]
    assert ims.copy_offsets(ims.ImageConfig((64, 48))) == [0]
