"""Vector-geometry (ASTRA-model) projector on the CPU: the geometry rows against the
reference's own genVectorsAstra (tests/golden/vecgeom.npz), analytic checks of the
oracle, and its agreement with the reference-pinned Python-projector oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import vecgeom as V
from vamtoolbox_b200.projector.Projector3DParallelCUDA import genVectorsAstra, parallel3d_vectors


def test_vectors_match_reference(golden):
    G = golden["vecgeom"]
    i = 0
    while f"v{i}_vectors" in G.files:
        mine = genVectorsAstra(G[f"v{i}_angles"], float(G[f"v{i}_incline"]))
        assert np.array_equal(mine, G[f"v{i}_vectors"]), i
        i += 1
    assert i >= 4
    mine = genVectorsAstra(np.array([0.0, 45.0, 100.0]), 10.0, cone_angle=5.0, distance_origin_source=250.0)
    assert np.array_equal(mine, G["cone_vectors"])


def test_parallel3d_rows():
    a = np.deg2rad([0.0, 30.0, 90.0])
    vec = parallel3d_vectors(a)
    assert np.allclose(vec[:, 0:3], np.stack([np.sin(a), -np.cos(a), 0 * a], 1))
    assert np.allclose(vec[:, 6:9], np.stack([np.cos(a), np.sin(a), 0 * a], 1))
    assert np.allclose(vec[:, 9:12], [[0, 0, 1]] * 3) and not vec[:, 3:6].any()


@pytest.mark.parametrize("incline", [0.0, 20.0, -35.0])
def test_voxel_projects_where_the_geometry_says(incline):
    """A single voxel forward-projects to the detector position the 3x3 solve gives."""
    shape = (24, 24, 16)
    vol = np.zeros(shape)
    idx = (15, 9, 6)
    vol[idx] = 1.0
    ang = np.array([0.0, 40.0, 115.0, 250.0])
    vec = genVectorsAstra(ang, incline)
    sino = V.forward(vol, vec, 24, 16)
    p = np.array(idx) + 0.5 - np.array(shape) / 2.0
    for a, q in enumerate(vec):
        M = np.stack([q[6:9], q[9:12], q[0:3]], axis=1)
        U, Vv, _ = np.linalg.solve(M, p - q[3:6])
        c, r = U + 12 - 0.5, Vv + 8 - 0.5
        plane = sino[:, a, :]
        cm = (plane.sum(1) * np.arange(24)).sum() / plane.sum()
        rm = (plane.sum(0) * np.arange(16)).sum() / plane.sum()
        assert abs(cm - c) < 0.35 and abs(rm - r) < 0.35, (a, cm, c, rm, r)


def test_backprojection_peaks_at_the_voxel():
    shape = (20, 20, 12)
    vec = genVectorsAstra(np.linspace(0, 180, 30, endpoint=False), 15.0)
    vol = np.zeros(shape)
    vol[12, 7, 5] = 1.0
    bp = V.backward(V.forward(vol, vec, 20, 12), vec, shape)
    assert np.unravel_index(np.argmax(bp), shape) == (12, 7, 5)


def _smooth_phantom(n, nz, seed=0):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[:n, :n].astype(float)
    vol = np.zeros((n, n, nz))
    for _ in range(5):
        cy, cx = rng.uniform(0.3 * n, 0.7 * n, 2)
        w = rng.uniform(0.08, 0.15) * n
        vol += rng.uniform(0.5, 1.0) * np.exp(-((y - cy) ** 2 + (x - cx) ** 2) / (2 * w * w))[:, :, None]
    return vol * np.linspace(0.5, 1.0, nz)[None, None, :]


def test_vertical_rays_agree_with_the_python_projector():
    """At zero inclination the model at angle theta + 90 degrees integrates along the
    Python projector's rays at theta (same ray and detector axes); its pixel c sits at
    Python bin c + 1/2 - (cos theta - sin theta) / 2 (centres (N-1)/2 versus N//2)."""
    n, nz = 48, 3
    vol = _smooth_phantom(n, nz)
    theta = np.linspace(0, 360, 24, endpoint=False)
    r1 = O.parallel_forward(vol, theta)                     # [n][nA][nz], pinned to the reference
    vec = parallel3d_vectors(np.deg2rad(theta + 90.0))
    astra = V.forward(vol, vec, n, nz)
    th = np.deg2rad(theta)
    res, ref = [], []
    for a in range(theta.size):
        jstar = np.arange(n) + 0.5 - 0.5 * (np.cos(th[a]) - np.sin(th[a]))
        for z in range(nz):
            res.append(astra[:, a, z])
            ref.append(np.interp(jstar, np.arange(n), r1[:, a, z]))
    res, ref = np.concatenate(res), np.concatenate(ref)
    assert np.linalg.norm(res - ref) / np.linalg.norm(ref) < 1e-2   # 0.4 %; other quarter turns: 57-79 %


def test_line_model_chord_lengths():
    """Rows of the line model hold intersection lengths: a ray through the image square
    collects exactly the length of its chord of that square."""
    n = 16
    M = V.line2d_matrix(n, n, np.array([0.0, 17.0, 45.0, 90.0, 133.0]), n)
    # a ray through the centre region crosses the whole 16 x 16 square
    for a, t in enumerate(np.deg2rad([0.0, 17.0, 45.0, 90.0, 133.0])):
        d = n // 2
        off = d - n / 2 + 0.5
        # chord of the square [-8, 8]^2 for the line at normal offset `off`
        dirv = np.array([np.sin(t), -np.cos(t)])
        p0 = np.array([np.cos(t), np.sin(t)]) * off
        s = []
        for k in range(2):
            if abs(dirv[k]) > 1e-12:
                s += sorted([(-8 - p0[k]) / dirv[k], (8 - p0[k]) / dirv[k]])
        lo = max(s[0::2]) if len(s) == 4 else s[0]
        hi = min(s[1::2]) if len(s) == 4 else s[1]
        assert abs(M[d * 5 + a].sum() - (hi - lo)) < 1e-9


def test_line_model_agrees_with_python_projector():
    """At equal angles ASTRA's 2-D frame (row 0 on top) and the reference-pinned Python
    projector integrate along the same rays; pixel c sits at Python bin
    c + 1/2 - (cos a - sin a)/2 (centres (N-1)/2 against N//2)."""
    n = 48
    img = _smooth_phantom(n, 1)[:, :, 0]
    theta = np.linspace(0, 360, 24, endpoint=False)
    r1 = O.parallel_forward(img[:, :, None], theta)[:, :, 0]
    lf = V.line2d_forward(img, theta, n)
    th = np.deg2rad(theta)
    res, ref = [], []
    for a in range(theta.size):
        jstar = np.arange(n) + 0.5 - 0.5 * (np.cos(th[a]) - np.sin(th[a]))
        res.append(lf[:, a])
        ref.append(np.interp(jstar, np.arange(n), r1[:, a]))
    res, ref = np.concatenate(res), np.concatenate(ref)
    assert np.linalg.norm(res - ref) / np.linalg.norm(ref) < 1e-2   # 0.43 %
