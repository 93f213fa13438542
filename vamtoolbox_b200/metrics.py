"""Dose-quality metrics: the reference's ``vamtoolbox.metrics`` (vamtoolbox/metrics.py:1-167).

Accept numpy arrays (reference semantics, float64) or CUDA tensors; the
volumetric error rate of a CUDA tensor is computed by the fused
vam_metric_ver kernel without leaving the device.
"""
from __future__ import annotations

import numpy as np


def _np(a):
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def calcCV(target, recon, layerwise=False):
    recon = _np(recon)
    g = target.gel_inds
    cv = np.std(recon[g]) / np.mean(recon[g])
    if not layerwise:
        return cv
    return np.full(recon.shape[2], cv)


def _device_metric(name, target, recon):
    """Whole-volume metric of a CUDA tensor by the fused reduction kernel (one float on the device,
    read back as a Python float)."""
    import torch

    from . import _lib

    x = recon.detach().to(torch.float32).contiguous()
    mask = torch.as_tensor(region_mask(target).reshape(x.shape), device=x.device)
    work = torch.empty(int(_lib.load().vam_reduce_workspace_bytes(x.numel())), dtype=torch.uint8, device=x.device)
    out = torch.empty(1, dtype=torch.float32, device=x.device)
    _lib.call(name, _lib.ptr(x), _lib.ptr(mask), x.numel(), _lib.ptr(out), _lib.ptr(work), work.numel(),
              _lib.stream_ptr(torch.cuda.current_stream(x.device)))
    return float(out.item())


def _on_cuda(recon):
    return getattr(recon, "is_cuda", False)


def _layer(mask, z):
    """The z-th slice of a gel / void mask.  (The reference's layerwise branches index each 2-D slice with
    the whole 3-D mask and raise IndexError, metrics.py:78-90, 118-127, 158-166; here they work.)"""
    mask = np.asarray(mask)
    return mask[:, :, z] if mask.ndim == 3 else mask


def calcVER(target, recon, layerwise=False):
    """#(void >= min(gel)) / (#gel + #void).  A CUDA tensor is reduced on the device (vam_metric_ver)."""
    if _on_cuda(recon) and not layerwise:
        return _device_metric("vam_metric_ver", target, recon)
    recon = _np(recon)
    gel, void = target.gel_inds, target.void_inds
    num = np.sum(gel[:]) + np.sum(void[:])
    if not layerwise:
        mn = np.min(recon[gel])
        return np.sum(recon[void] >= mn) / num
    out = np.zeros(recon.shape[2])
    for z in range(recon.shape[2]):
        s = recon[:, :, z]
        out[z] = np.sum(s[_layer(void, z)] >= np.min(s[_layer(gel, z)])) / num
    return out


def calcPW(target, recon, layerwise=False):
    recon = _np(recon)
    gel, void = target.gel_inds, target.void_inds
    if not layerwise:
        return np.max(recon[void]) - np.min(recon[gel])
    out = np.zeros(recon.shape[2])
    for z in range(recon.shape[2]):
        s = recon[:, :, z]
        out[z] = np.max(s[_layer(void, z)]) - np.min(s[_layer(gel, z)])
    return out


def calcIPDR(target, recon, layerwise=False):
    """max(gel) - min(gel) (metrics.py:130-156).  A CUDA tensor is reduced on the device
    (vam_metric_ipdr)."""
    if _on_cuda(recon) and not layerwise:
        return _device_metric("vam_metric_ipdr", target, recon)
    recon = _np(recon)
    gel = target.gel_inds
    if not layerwise:
        return np.max(recon[gel]) - np.min(recon[gel])
    out = np.zeros(recon.shape[2])
    for z in range(recon.shape[2]):
        s, gz = recon[:, :, z], _layer(gel, z)
        out[z] = np.max(s[gz]) - np.min(s[gz])
    return out


def region_mask(target):
    """uint8 mask: 1 gel, 2 void, 0 outside the circle (used by the device VER)."""
    m = np.zeros(np.shape(target.gel_inds), dtype=np.uint8)
    m[target.gel_inds] = 1
    m[target.void_inds] = 2
    return m


def ver_device(x, mask_dev, out, work):
    """VER of CUDA tensor x into out[0] (device), mask_dev from region_mask."""
    import torch

    from . import _lib

    _lib.call("vam_metric_ver", _lib.ptr(x), _lib.ptr(mask_dev), x.numel(), _lib.ptr(out), _lib.ptr(work),
              work.numel(), _lib.stream_ptr(torch.cuda.current_stream(x.device)))
    return out
