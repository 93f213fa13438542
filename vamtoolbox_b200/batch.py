"""Many projector calls over many plans in persistent launches.

``ProjectionBatch`` binds ``vam_batch_*``: a list of (plan, op, input, output)
calls -- targets of uneven size, 2-D slices next to 3-D volumes, different
angle counts -- runs as one persistent kernel per kernel-body family present
(each compiled with only that family's bodies), whose CTAs take the calls'
blocks from a device work queue, largest call first.  Each call computes
exactly what the plan's own forward / backward_ref / adjoint computes
(bit-identical), so a batch is a drop-in for running the targets one at a
time through the reference's per-target projector calls
(vamtoolbox/projector/Projector3DParallel.py:113-207).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib

OPS = {"forward": _lib.OP_FORWARD, "backward": _lib.OP_BACKWARD_REF, "backward_ref": _lib.OP_BACKWARD_REF,
       "adjoint": _lib.OP_ADJOINT}


class ProjectionBatch:
    """A reusable work queue on one device.

    ``submit(work)`` runs the calls on the current stream (capturable in a
    CUDA graph: the call descriptions travel in the launch parameters);
    ``prepare(work)`` only validates a list.  Calls of one batch run
    concurrently: no call may read another's output, and a plan appears at
    most once as a forward (its mask-mode scratch volume is per plan).
    """

    def __init__(self, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("vamtoolbox_b200 batches need a CUDA device (no CPU fallback)")
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        h = ctypes.c_void_p()
        _lib.call("vam_batch_create", self.device.index, ctypes.byref(h))
        self._h = h
        self._arr = None
        self._keep = None

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.load().vam_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _works(self, work):
        items = []
        keep = []
        for plan, op, x, y in work:
            if op not in OPS:
                raise ValueError(f"unknown op {op!r}; expected one of {sorted(OPS)}")
            fwd = OPS[op] == _lib.OP_FORWARD
            shape_in, shape_out = (plan.shape_vol, plan.shape_sino) if fwd else (plan.shape_sino, plan.shape_vol)
            plan._check(x, shape_in, f"batch {op} input")
            plan._check(y, shape_out, f"batch {op} output")
            if plan.device != self.device:
                raise ValueError(f"plan on {plan.device}, batch on {self.device}")
            if OPS[op] == _lib.OP_ADJOINT and not plan._adj_ready and not torch.cuda.is_current_stream_capturing():
                plan.prepare_adjoint()
            items.append(_lib.Work(plan.handle.value, OPS[op], x.data_ptr(), y.data_ptr()))
            keep.append((plan, x, y))
        arr = (_lib.Work * len(items))(*items)
        return arr, keep

    def prepare(self, work):
        arr, keep = self._works(work)
        with torch.cuda.device(self.device):
            _lib.call("vam_batch_prepare", self._h, arr, len(keep), _lib.stream_ptr(torch.cuda.current_stream(self.device)))
        self._arr, self._keep = arr, keep

    def submit(self, work):
        arr, keep = self._works(work)
        with torch.cuda.device(self.device):
            _lib.call("vam_batch_submit", self._h, arr, len(keep), _lib.stream_ptr(torch.cuda.current_stream(self.device)))
        self._arr, self._keep = arr, keep

    def info(self):
        vb, ctas = ctypes.c_int64(), ctypes.c_int32()
        _lib.call("vam_batch_info", self._h, ctypes.byref(vb), ctypes.byref(ctas))
        return {"virtual_blocks": int(vb.value), "ctas": int(ctas.value)}
