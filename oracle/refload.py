"""Load the reference VAMToolbox's hot-path modules in this container.

TEST INFRASTRUCTURE ONLY (used by tests/golden/make_golden.py to generate
golden vectors; never imported by the product package or at run time on a
GPU host, where the reference tree does not exist).

``import vamtoolbox`` fails here: its package __init__ pulls in plotting,
OpenGL voxelisation and DLP playback (vamtoolbox/__init__.py:1-16), and
astra / skimage / matplotlib are not installed.  This loader registers
synthetic package modules for ``vamtoolbox`` and its sub-packages (so their
__init__ files are bypassed), stubs matplotlib and astra, and installs a
restated ``skimage.transform._warps.warp`` (order-1 bilinear, constant mode,
cval 0, inverse map (col, row, 1) @ M^T) so the reference's own projector code
runs around it.  The stubbed warp is the one restated piece; everything else
executed is the reference's code.
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np

REF = os.environ.get("VAM_REFERENCE_ROOT", "/root/reference")


def available() -> bool:
    return os.path.isdir(os.path.join(REF, "vamtoolbox"))


def _stub(name, **attrs):
    m = types.ModuleType(name)
    m.__file__ = "<stub>"
    m.__dict__.update(attrs)
    sys.modules[name] = m
    return m


class _Anything:
    def __getattr__(self, k):
        return _Anything()

    def __call__(self, *a, **k):
        return _Anything()


def restated_warp(image, inverse_map, clip=True, preserve_range=False, **_):
    """skimage.transform.warp(image, 3x3 matrix) for order=1, mode='constant', cval=0.

    Bilinear with floor/ceil neighbours and zero outside, coordinates
    computed as (M00*col + M01*row) + M02 in float64.  Integer images are
    scaled by 1/max(dtype) like skimage's img_as_float (irrelevant to the
    callers, which only test > 0).
    """
    img = np.asarray(image)
    if np.issubdtype(img.dtype, np.integer) and not preserve_range:
        img = img.astype(np.float64) / np.iinfo(img.dtype).max
    img = img.astype(np.float64)
    rows, cols = img.shape
    M = np.asarray(inverse_map, dtype=np.float64)
    rr, cc = np.mgrid[:rows, :cols].astype(np.float64)
    cin = (M[0, 0] * cc + M[0, 1] * rr) + M[0, 2]
    rin = (M[1, 0] * cc + M[1, 1] * rr) + M[1, 2]
    minr, minc = np.floor(rin).astype(np.int64), np.floor(cin).astype(np.int64)
    maxr, maxc = np.ceil(rin).astype(np.int64), np.ceil(cin).astype(np.int64)
    dr, dc = rin - minr, cin - minc

    def px(r, c):
        ok = (r >= 0) & (r < rows) & (c >= 0) & (c < cols)
        out = np.zeros_like(rin)
        out[ok] = img[r[ok], c[ok]]
        return out

    top = (1 - dc) * px(minr, minc) + dc * px(minr, maxc)
    bottom = (1 - dc) * px(maxr, minc) + dc * px(maxr, maxc)
    return (1 - dr) * top + dr * bottom


_loaded = None


def load():
    """Return the reference ``vamtoolbox`` package object (hot-path modules only)."""
    global _loaded
    if _loaded is not None:
        return _loaded
    if not available():
        raise RuntimeError(f"reference tree not found at {REF}")
    # numpy 2 removed np.product, which BCLP.py:540 and PM.py:307,371 still
    # call; alias it to np.prod (identical semantics) for the reference run.
    if not hasattr(np, "product"):
        np.product = np.prod
    import scipy.ndimage  # noqa: F401  (import heavy deps before stubbing)
    import torch  # noqa: F401

    if "matplotlib" not in sys.modules:
        mpl = _stub("matplotlib")
        plt = _stub("matplotlib.pyplot")
        plt.__getattr__ = lambda k: _Anything()
        mpl.pyplot = plt
        _stub("mpl_toolkits")
        _stub("mpl_toolkits.axes_grid1", make_axes_locatable=lambda *a, **k: None)
    _stub("astra")
    _stub("skimage")
    _stub("skimage.transform")
    _stub("skimage.transform._warps", warp=restated_warp)
    pkg = types.ModuleType("vamtoolbox")
    pkg.__path__ = [os.path.join(REF, "vamtoolbox")]
    pkg.__file__ = os.path.join(REF, "vamtoolbox", "__init__.py")
    sys.modules["vamtoolbox"] = pkg
    for sub in ("util", "projector", "optimizer"):
        m = types.ModuleType("vamtoolbox." + sub)
        m.__path__ = [os.path.join(REF, "vamtoolbox", sub)]
        sys.modules["vamtoolbox." + sub] = m
        setattr(pkg, sub, m)
    import importlib

    pkg.util.data = importlib.import_module("vamtoolbox.util.data")
    for name in ("geometry", "metrics", "response", "medium", "projectorconstructor", "optimize"):
        if name == "projectorconstructor":
            pass
        setattr(pkg, name, importlib.import_module("vamtoolbox." + name))
    pkg.projector.Projector3DParallel = importlib.import_module("vamtoolbox.projector.Projector3DParallel")
    pkg.projector.Projector2DParallel = importlib.import_module("vamtoolbox.projector.Projector2DParallel")
    pkg.projector.pyTorchRayTrace = importlib.import_module("vamtoolbox.projector.pyTorchRayTrace")
    pkg.projector.pyTorchAlgebraicPropagation = importlib.import_module("vamtoolbox.projector.pyTorchAlgebraicPropagation")
    for opt in ("CAL", "OSMO", "BCLP", "PM", "FBP"):
        setattr(pkg.optimizer, opt, importlib.import_module("vamtoolbox.optimizer." + opt))
    # frame output (cv2 / dill / PIL are present here; its preview player is not imported)
    pkg.imagesequence = importlib.import_module("vamtoolbox.imagesequence")
    _loaded = pkg
    return pkg


class _NoInferenceMode:
    """Stands in for torch.inference_mode while a module is imported: as a decorator it returns the
    function unchanged, as a context manager it does nothing, so the reference's tracer records
    autograd graphs."""

    def __init__(self, *a, **k):
        pass

    def __call__(self, fn):
        return fn

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def load_autograd_tracer():
    """Second copies of the reference's pyTorchRayTrace.py and medium.py, imported with
    torch.inference_mode neutralised (their decorators are applied at import), so gradients can be
    taken through the reference's own ray tracer.  Returns (tracer module, medium module)."""
    import importlib.util

    import torch

    load()
    orig = torch.inference_mode
    torch.inference_mode = _NoInferenceMode
    try:
        mods = []
        for name, rel in (("vamtoolbox.projector._rt_autograd", "projector/pyTorchRayTrace.py"),
                          ("vamtoolbox._medium_autograd", "medium.py")):
            spec = importlib.util.spec_from_file_location(name, os.path.join(REF, "vamtoolbox", rel))
            m = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(m)
            mods.append(m)
    finally:
        torch.inference_mode = orig
    return mods[0], mods[1]


def fresh_options(pkg, **kw):
    """Options(...) with the class-level default dicts restored first.

    The reference mutates Options' class-level defaults on every construction
    (vamtoolbox/optimize.py:119-126), so kwargs leak between instances; the
    snapshot below keeps each golden case independent.
    """
    O = pkg.optimize.Options
    if not hasattr(O, "_golden_snapshot"):
        O._golden_snapshot = {k: dict(v) for k, v in vars(O).items() if k.startswith("_Options__default")}
    for k, v in O._golden_snapshot.items():
        getattr(O, k).clear()
        getattr(O, k).update(v)
    return O(**kw)
