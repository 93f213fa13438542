"""The C-ABI library loads and exports every function include/vam.h declares (CPU only)."""
import ctypes
import re
from pathlib import Path

from vamtoolbox_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    src = (ROOT / "include" / "vam.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(vam_[a-z_0-9]+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "vam_parallel_forward" in names and "vam_ray_deposit" in names
    assert len(names) >= 25


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_functions()) == set(_lib.exported_symbols())


def test_version_and_error_string_without_gpu():
    assert _lib.version().startswith("vamcore")
    lib = _lib.load()
    assert lib.vam_last_error_string() is not None


def test_argument_errors_are_reported_without_touching_the_gpu():
    lib = _lib.load()
    h = ctypes.c_void_p()
    code = lib.vam_parallel_plan_create(None, ctypes.byref(h))
    assert code == _lib.VAM_ERR_ARG
    assert b"null" in lib.vam_last_error_string()
    ang = (ctypes.c_double * 3)(0.0, 1.0, 2.0)
    geom = _lib.ParallelGeom(16, 12, 1, 3, ang, 0)   # non-square slice
    assert lib.vam_parallel_plan_create(ctypes.byref(geom), ctypes.byref(h)) == _lib.VAM_ERR_SHAPE
    geom = _lib.ParallelGeom(16, 16, 0, 3, ang, 0)
    assert lib.vam_parallel_plan_create(ctypes.byref(geom), ctypes.byref(h)) == _lib.VAM_ERR_SHAPE
    assert lib.vam_reduce(None, 10, 0, None, None, 0, None) == _lib.VAM_ERR_ARG
    assert lib.vam_reduce_workspace_bytes(1 << 20) > 0
