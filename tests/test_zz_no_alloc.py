"""vam_reduce_noalloc: the reduction for callers that cannot allocate device memory.

Some callers can't call cudaMalloc: printer hosts that reserve all device
memory for their projection buffers before a print starts (an allocation
would fail) and must not trigger cudaMalloc's implicit synchronisation during
exposure, and plug-ins that are handed fixed buffers and have no allocator.  This entry point keeps its scratch in a
static device array inside the library instead of a caller workspace.  The
test calls it through the C ABI and checks it against the workspace-based
vam_reduce and against a float64 numpy reduction of the same data, twice in
a row on different data (the shared scratch keeps the previous call's
contents), and checks that sizes above its stated maximum are rejected before
anything is launched.  It lives in a file pytest collects last.
"""
import ctypes

import numpy as np
import pytest
import torch

from vamtoolbox_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_N = 4096 * 2048  # 4096 static partials, one per 2048 inputs


def _call_noalloc(x, op, out):
    lib = _lib.load()
    return lib.vam_reduce_noalloc(_lib.ptr(x), x.numel(), op, _lib.ptr(out), _lib.stream_ptr())


@pytest.mark.parametrize("n", [1, 777, 100_003, MAX_N])
def test_noalloc_reduce_matches_workspace_reduce_on_two_calls(n):
    lib = _lib.load()
    work = torch.empty(int(lib.vam_reduce_workspace_bytes(n)), dtype=torch.uint8, device="cuda")
    rng = np.random.default_rng(n)
    for call in range(2):
        xh = rng.standard_normal(n).astype(np.float32)
        x = torch.as_tensor(xh, device="cuda")
        x64 = xh.astype(np.float64)
        exact = {_lib.RED_MAX: float(x64.max()), _lib.RED_MIN: float(x64.min()), _lib.RED_SUM: float(x64.sum())}
        for op in (_lib.RED_MAX, _lib.RED_MIN, _lib.RED_SUM):
            ref = torch.full((1,), float("nan"), device="cuda")
            got = torch.full((1,), float("nan"), device="cuda")
            _lib.call("vam_reduce", _lib.ptr(x), n, op, _lib.ptr(ref), _lib.ptr(work), work.numel(),
                      _lib.stream_ptr())
            assert _call_noalloc(x, op, got) == _lib.VAM_OK
            torch.cuda.synchronize()
            r, g = float(ref.item()), float(got.item())
            assert np.isfinite(g)
            assert abs(g - r) <= 1e-6 * max(1.0, abs(r)), (call, op, g, r)
            # independent check: max and min are exact; the sum is accumulated in float64 and rounded
            # once to float32, so it lies within one float32 ulp of numpy's float64 sum
            if op == _lib.RED_SUM:
                assert abs(g - exact[op]) <= 2 ** -23 * max(abs(exact[op]), 1.0), (call, g, exact[op])
            else:
                assert g == exact[op], (call, op, g, exact[op])


def test_noalloc_reduce_rejects_sizes_above_its_maximum():
    lib = _lib.load()
    x = torch.zeros(16, device="cuda")
    out = torch.zeros(1, device="cuda")
    code = lib.vam_reduce_noalloc(_lib.ptr(x), MAX_N + 1, _lib.RED_SUM, _lib.ptr(out), _lib.stream_ptr())
    assert code == _lib.VAM_ERR_SHAPE
    msg = lib.vam_last_error_string().decode()
    assert "exceeds the maximum of 8388608 elements" in msg
