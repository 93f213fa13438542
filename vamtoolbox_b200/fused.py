"""Device-resident optimizer building blocks over the fused kernels (csrc/optim.cu).

A :class:`Workspace` owns the reduction scratch and small device scalars so
that an optimizer iteration issues only stream-ordered kernel launches (no
allocation, no host synchronisation) and can be captured once in a CUDA
graph with :func:`capture` and replayed.
"""
from __future__ import annotations

import ctypes
import gc

import numpy as np
import torch

from . import _lib


class Workspace:
    def __init__(self, device):
        self.device = torch.device(device)
        nbytes = int(_lib.load().vam_reduce_workspace_bytes(1 << 30))
        self.work = torch.empty(nbytes, dtype=torch.uint8, device=self.device)

    def stream(self):
        return _lib.stream_ptr(torch.cuda.current_stream(self.device))

    def scalar(self, n=1):
        return torch.zeros(n, dtype=torch.float32, device=self.device)

    # reductions -------------------------------------------------------------
    def reduce(self, x, op, out):
        _lib.call("vam_reduce", _lib.ptr(x), x.numel(), op, _lib.ptr(out), _lib.ptr(self.work), self.work.numel(),
                  self.stream())
        return out

    def max(self, x, out):
        return self.reduce(x, _lib.RED_MAX, out)

    def ver(self, x, mask, out):
        _lib.call("vam_metric_ver", _lib.ptr(x), _lib.ptr(mask), x.numel(), _lib.ptr(out), _lib.ptr(self.work),
                  self.work.numel(), self.stream())
        return out

    # elementwise ------------------------------------------------------------
    def scale(self, x, s, floor=None):
        _lib.call("vam_scale_by_device", _lib.ptr(x), _lib.ptr(s), x.numel(), int(floor is not None),
                  float(floor or 0.0), self.stream())
        return x

    def cal_threshold(self, x, xmax, target, d_h, g, out):
        _lib.call("vam_cal_threshold", _lib.ptr(x), _lib.ptr(xmax), _lib.ptr(target), x.numel(), float(d_h), float(g),
                  _lib.ptr(out), self.stream())
        return out

    def cal_update(self, b, db, db_prev, lr, momentum, it):
        _lib.call("vam_cal_sino_update", _lib.ptr(b), _lib.ptr(db), _lib.ptr(db_prev), b.numel(), float(lr),
                  float(momentum), int(it), self.stream())
        return b

    def osmo_model(self, xm, x, xmax, mask, gel, d):
        _lib.call("vam_osmo_model_update", _lib.ptr(xm), _lib.ptr(x), _lib.ptr(xmax), _lib.ptr(mask), xm.numel(),
                  int(gel), float(d), self.stream())
        return xm

    def bclp_dose_pass(self, dose, target, prm, mapped, operand, stats):
        _lib.call("vam_bclp_dose_pass", _lib.ptr(dose), _lib.ptr(target), dose.numel(), ctypes.byref(prm),
                  _lib.ptr(mapped), _lib.ptr(operand), _lib.ptr(stats), _lib.ptr(self.work), self.work.numel(),
                  self.stream())

    def bclp_update(self, g, grad, lr, p, q, lo, hi, stats):
        has_hi = hi is not None
        _lib.call("vam_bclp_sino_update", _lib.ptr(g), _lib.ptr(grad), g.numel(), float(lr), float(p), float(q),
                  float(lo if lo is not None else -3.0e38), float(hi if has_hi else 0.0), int(has_hi), _lib.ptr(stats),
                  self.stream())

    def append(self, src, arr, counter):
        n = src.numel()
        _lib.call("vam_append", _lib.ptr(src), n, _lib.ptr(arr), _lib.ptr(counter), arr.numel() // n, self.stream())


def bclp_params(response_model, eps, weight, p, device, keep):
    """vam_bclp_params for a response model: interpolation tables on the device, or the closed form
    of an analytical generalised-logistic / linear / identity model (evaluated in float64 per voxel)."""
    prm = _lib.BclpParams()
    rm = response_model
    if rm.type == "interpolation":
        f, m, dm, f0, inv_step = rm.device_tables(device)
        prm.table_f, prm.table_map, prm.table_dmap = f.data_ptr(), m.data_ptr(), dm.data_ptr()
        prm.n_table = f.numel()
        prm.table_f0, prm.table_inv_step = f0, inv_step
        prm.response = _lib.RESP_TABLE
        keep += [f, m, dm]
    elif rm.form == "gen_log_fun":
        q = rm.params
        prm.response = _lib.RESP_GLF
        prm.resp_A, prm.resp_K, prm.resp_B = float(q["A"]), float(q["K"]), float(q["B"])
        prm.resp_M, prm.resp_nu = float(q["M"]), float(q["nu"])
    elif rm.form == "linear":
        prm.response = _lib.RESP_LINEAR
        prm.resp_M, prm.resp_C = float(rm.params["M"]), float(rm.params["C"])
    elif rm.form == "identity":
        prm.response = _lib.RESP_IDENTITY
    else:
        raise NotImplementedError(f"response model {rm.type}/{rm.form} has no device form")
    prm.p = float(p)
    if isinstance(eps, torch.Tensor):
        keep.append(eps)
        prm.eps_dev, prm.eps = eps.data_ptr(), 0.0
    else:
        prm.eps = float(eps)
    if isinstance(weight, torch.Tensor):
        keep.append(weight)
        prm.weight_dev, prm.weight = weight.data_ptr(), 0.0
    else:
        prm.weight = float(weight)
    return prm


def capture(fn, device):
    """Capture fn() into a CUDA graph without executing it.

    fn must only issue stream-ordered kernel launches on the current stream
    (the C-ABI calls of this package) and no host synchronisation; its
    buffers must stay alive as long as the graph.  Replay with graph.replay().
    """
    device = torch.device(device)
    g = torch.cuda.CUDAGraph(keep_graph=True)  # keeps the cudaGraph_t readable (graph_kernel_nodes)
    s = _capture_stream(device)
    # capture_begin / capture_end directly: the torch.cuda.graph context manager also runs a Python
    # garbage collection and empties the allocator cache on entry (tens of ms per capture), which the
    # captured launches here do not need (they allocate nothing)
    s.wait_stream(torch.cuda.current_stream(device))
    # no garbage collection while capturing: a collected object that owns device memory (a plan released
    # earlier) would free it inside the capture, which invalidates the graph
    gc_on = gc.isenabled()
    gc.disable()
    try:
        with torch.cuda.stream(s):
            g.capture_begin(capture_error_mode="global")
            try:
                fn()
            finally:
                g.capture_end()
    finally:
        if gc_on:
            gc.enable()
    torch.cuda.current_stream(device).wait_stream(s)
    g.instantiate()
    return g


_CAPTURE_STREAMS = {}


def _capture_stream(device):
    """One side stream per device for captures (a capture may not run on the legacy default stream)."""
    key = str(device)
    if key not in _CAPTURE_STREAMS:
        _CAPTURE_STREAMS[key] = torch.cuda.Stream(device=device)
    return _CAPTURE_STREAMS[key]


def to_host_f64(*tensors):
    """float64 host arrays of device tensors: converted on the device and copied into page-locked host
    buffers from torch's caching host allocator, one synchronisation for all.  Returning arrays that
    view page-locked memory avoids faulting in fresh pageable memory for every result (a pageable
    download of a 256^3 dose and sinogram took ~150 ms, a page-locked one from the cache ~7 ms)."""
    outs = []
    for t in tensors:
        d = t.detach().to(torch.float64)
        h = torch.empty(d.shape, dtype=torch.float64, pin_memory=True)
        h.copy_(d, non_blocking=True)
        outs.append(h)
    torch.cuda.current_stream(tensors[0].device).synchronize()
    return [h.numpy() for h in outs]


_COPY_POOL = None


def _copy_pool():
    global _COPY_POOL
    if _COPY_POOL is None:
        import concurrent.futures
        import os

        _COPY_POOL = concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1)))
    return _COPY_POOL


def to_device_f64(array, device):
    """A host array as a float64 device tensor, staged through a page-locked buffer of torch's caching
    host allocator that several threads fill in chunks (numpy releases the GIL for plain copies); each
    chunk's asynchronous copy on the current stream is issued as soon as that chunk is staged, so the
    host copy and the transfer overlap.  A pageable upload of a 256^3 float64 target ran at about
    10 GB/s (13 ms), staged then copied whole about 7 ms; the allocator keeps the staging block alive
    until the copies have run."""
    a = np.ascontiguousarray(array, dtype=np.float64)
    if a.nbytes < (8 << 20):
        return torch.as_tensor(a).to(device)
    h = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    d = torch.empty(a.shape, dtype=torch.float64, device=device)
    hf, df = h.view(-1), d.view(-1)
    dst, src = h.numpy().reshape(-1), a.reshape(-1)
    pool = _copy_pool()
    step = -(-src.size // (4 * pool._max_workers))
    spans = [(lo, min(lo + step, src.size)) for lo in range(0, src.size, step)]
    staged = [pool.submit(np.copyto, dst[lo:hi], src[lo:hi]) for lo, hi in spans]
    for (lo, hi), f in zip(spans, staged):
        f.result()
        df[lo:hi].copy_(hf[lo:hi], non_blocking=True)
    return d


def graph_kernel_nodes(graph):
    """Number of kernel nodes in a captured torch CUDA graph (the launches one replay issues),
    read back through the CUDA runtime; None when the graph cannot be inspected."""
    try:
        from cuda.bindings import runtime as rt

        h = rt.cudaGraph_t(init_value=int(graph.raw_cuda_graph()))
        err, _, num = rt.cudaGraphGetNodes(h, numNodes=0)
        if int(err) != 0:
            return None
        err, nodes, num = rt.cudaGraphGetNodes(h, numNodes=num)
        if int(err) != 0:
            return None
        kernel = rt.cudaGraphNodeType.cudaGraphNodeTypeKernel
        count = 0
        for nd in nodes[:num]:
            e2, t = rt.cudaGraphNodeGetType(nd)
            if int(e2) == 0 and t == kernel:
                count += 1
        return count
    except Exception:
        return None
