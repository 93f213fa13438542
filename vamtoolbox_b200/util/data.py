"""Array helpers of the reference's ``vamtoolbox.util.data`` (vamtoolbox/util/data.py).

Host (numpy) versions keep the reference's semantics, including its in-place
writes (``clipToCircle`` modifies and returns its argument); ``*_t`` variants
operate on torch tensors on the device.  The Fourier filters run once per
optimisation at initialisation; the sinogram filter has a device version
(batched FFT along the detector axis, ``filterSinogram_t``).
"""
from __future__ import annotations

import numpy as np
import scipy.fft
from scipy.fft import fft, fft2, ifft, ifft2


def sigmoid(x, g):
    """1 / (1 + exp(-x / g)) (util/data.py:9-11)."""
    return (1 / (1 + np.exp(-x * (1 / g)))).astype(float)


def _circle_outside(ny, nx):
    cy, cx = np.meshgrid(np.linspace(-1, 1, ny), np.linspace(-1, 1, nx))
    return cx ** 2 + cy ** 2 > 1


def clipToCircle(x):
    """Zero everything outside the inscribed circle, in place (util/data.py:14-40)."""
    out = _circle_outside(x.shape[0], x.shape[1])
    if x.ndim == 2:
        x[out] = 0
    else:
        x[np.broadcast_to(out[..., np.newaxis], x.shape)] = 0
    return x


def circle_inside_mask(ny, nx):
    """Boolean [ny, nx] mask of the pixels clipToCircle keeps."""
    return ~_circle_outside(ny, nx)


def _osmo_filter(n_y, n_x, filter_name):
    """The radial 2-D frequency filter of filterTargetOSMO (util/data.py:43-113), n_y x n_x, float64."""
    filter_types = ("ram-lak", "shepp-logan", "cosine", "hamming", "hanning", None)
    if filter_name not in filter_types:
        raise ValueError("Unknown filter: %s" % filter_name)
    f_y, f_x = np.meshgrid(np.linspace(-1, 1, n_y), np.linspace(-1, 1, n_x), indexing="ij")
    f = np.sqrt(f_x ** 2 + f_y ** 2)
    filt = np.real(f)
    if filter_name == "shepp-logan":
        omega = np.pi / 2 * f
        nz = omega != 0
        filt[nz] *= np.sin(omega[nz]) / omega[nz]
    elif filter_name == "cosine":
        filt *= np.cos(np.pi / 2 * f)
    elif filter_name == "hamming":
        w = np.abs(np.hamming(n_x))
        filt *= np.abs(np.sqrt(np.outer(w, w)))
    elif filter_name == "hanning":
        w = np.abs(np.hanning(n_x))
        filt *= np.abs(np.sqrt(np.outer(w, w)))
    return filt


def filterTargetOSMO(x, filter_name):
    """Radial 2-D Fourier filter of each z slice (util/data.py:43-113)."""
    if filter_name is None or filter_name.lower() == "none":
        return x
    filt = _osmo_filter(x.shape[0], x.shape[1], filter_name)
    X = scipy.fft.fftshift(fft2(x, axes=(0, 1)), axes=(0, 1))
    if x.ndim == 2:
        out = ifft2(scipy.fft.ifftshift(X * filt, axes=(0, 1)), axes=(0, 1))
    else:
        out = ifft2(scipy.fft.ifftshift(X * filt[:, :, np.newaxis], axes=(0, 1)), axes=(0, 1))
    return out.astype(float)


def filterTargetOSMO_t(x, filter_name):
    """Device version of filterTargetOSMO for a [nY, nX] or [nY, nX, nZ] torch tensor: float64 cuFFT
    (through torch.fft) of every slice, the same filter, the real part; returned in x's dtype."""
    import torch

    if filter_name is None or filter_name.lower() == "none":
        return x
    filt = torch.as_tensor(_osmo_filter(x.shape[0], x.shape[1], filter_name), device=x.device, dtype=torch.float64)
    if x.ndim == 3:
        filt = filt[:, :, None]
    X = torch.fft.fftshift(torch.fft.fft2(x.to(torch.float64), dim=(0, 1)), dim=(0, 1))
    out = torch.fft.ifft2(torch.fft.ifftshift(X * filt, dim=(0, 1)), dim=(0, 1)).real
    return out.to(x.dtype).contiguous()


def filterTargetBCLP(real_space_array, filter_name):
    """Radial Fourier filter of each z slice for BCLP targets (util/data.py:116-196): |f| on the
    fftfreq grid, centred, with the window of the named filter; the Shepp-Logan and cosine windows are
    evaluated on the uncentred frequencies and multiplied into the centred filter, as the reference
    does.  The first two axes must have equal length."""
    filter_types = ("ram-lak", "shepp-logan", "cosine", "hamming", "hanning", None)
    if filter_name not in filter_types:
        raise ValueError("Unknown filter: %s" % filter_name)
    if filter_name is None or filter_name.lower() == "none":
        return real_space_array
    n_x, n_y = real_space_array.shape[0], real_space_array.shape[1]
    assert n_x == n_y, "The first two dimensions of the real space array must have the same number of elements."
    f_x, f_y = np.meshgrid(scipy.fft.fftfreq(n_x), scipy.fft.fftfreq(n_y), indexing="ij")
    f_radial = np.sqrt(f_x ** 2 + f_y ** 2)
    filt = scipy.fft.fftshift(f_radial)
    if filter_name == "shepp-logan":
        omega = np.pi / 2 * f_radial
        nz = omega != 0
        filt[nz] *= np.sin(omega[nz]) / omega[nz]
    elif filter_name == "cosine":
        filt *= np.cos(np.pi / 2 * f_radial)
    elif filter_name in ("hamming", "hanning"):
        w = np.abs(np.hamming(n_x) if filter_name == "hamming" else np.hanning(n_x))
        filt *= np.abs(np.sqrt(np.outer(w, w)))
    X = scipy.fft.fftshift(fft2(real_space_array, axes=(0, 1)), axes=(0, 1))
    f = filt if real_space_array.ndim == 2 else filt[:, :, np.newaxis]
    return np.real(ifft2(scipy.fft.ifftshift(X * f, axes=(0, 1)), axes=(0, 1))).astype(float)


def filterTarget(real_space_array, filter_name):
    """Each z slice filtered with the 2-D radial extension of the 1-D sinogram filter
    (util/data.py:199-300): the slices zero-padded in x / y (centred) to the next power of two, at least
    64; the 1-D filter of that length (_get_fourier_filter) interpolated linearly at every radial
    frequency |f| (zero beyond its last frequency); the product with the slices' 2-D FFT transformed
    back and cropped to the input size."""
    n_x, n_y = real_space_array.shape[0], real_space_array.shape[1]
    assert n_x == n_y, "The first two dimensions of the real space array must have the same number of elements."
    n_p = max(64, int(2 ** np.ceil(np.log2(n_x))))
    before, after = int(np.ceil((n_p - n_x) / 2)), int(np.floor((n_p - n_x) / 2))
    pad = ((before, after), (before, after)) + (() if real_space_array.ndim == 2 else ((0, 0),))
    padded = np.pad(real_space_array, pad, mode="constant", constant_values=0)
    f1 = np.squeeze(_get_fourier_filter(n_p, filter_name))
    freq = scipy.fft.fftfreq(n_p)
    order = freq.argsort()
    f_x, f_y = np.meshgrid(freq, freq, indexing="ij")
    filt = np.interp(np.sqrt(f_x ** 2 + f_y ** 2), np.sort(freq), f1[order], left=0, right=0)
    if real_space_array.ndim > 2:
        filt = filt[:, :, np.newaxis]
    out = np.real(ifft2(fft2(padded, axes=(0, 1)) * filt, axes=(0, 1))).astype(float)
    return out[before:, before:] if after == 0 else out[before:-after, before:-after]


def histogramEqualization(x, bit_depth, output_dtype=float):
    """Contrast stretch of util/data.py:471-492: x scaled by max / (99th - 1st percentile), then values
    at or above the 99th percentile set to 1 and at or below the 1st to 0 (bit_depth and output_dtype
    are accepted and unused, as in the reference)."""
    mx = np.amax(x)
    p01, p99 = np.percentile(x, 1), np.percentile(x, 99)
    y = x * (mx / (p99 - p01))
    y = np.where(y >= p99, 1, y)
    return np.where(y <= p01, 0, y)


def _get_fourier_filter(size, filter_name):
    """Ram-Lak family filter built from its spatial form (util/data.py:373-438; Kak & Slaney ch. 3 eq. 61)."""
    n = np.concatenate((np.arange(1, size / 2 + 1, 2, dtype=int), np.arange(size / 2 - 1, 0, -2, dtype=int)))
    f = np.zeros(size)
    f[0] = 0.25
    f[1::2] = -1 / (np.pi * n) ** 2
    filt = 2 * np.real(fft(f))
    if filter_name == "shepp-logan":
        omega = np.pi * scipy.fft.fftfreq(size)[1:]
        filt[1:] *= np.sin(omega) / omega
    elif filter_name == "cosine":
        filt *= scipy.fft.fftshift(np.sin(np.linspace(0, np.pi, size, endpoint=False)))
    elif filter_name == "hamming":
        filt *= scipy.fft.fftshift(np.hamming(size))
    elif filter_name == "hanning":
        filt *= scipy.fft.fftshift(np.hanning(size))
    elif filter_name == "ram-lak_freq":
        filt /= (np.pi / 4) ** 2
    elif filter_name == "ram-lak_scikit":
        filt *= np.pi / 2
    elif filter_name is None or filter_name.lower() == "none":
        filt[:] = 1
    return filt[:, np.newaxis]


_SINO_FILTERS = ("ram-lak", "shepp-logan", "cosine", "hamming", "hanning", "ram-lak_freq", "ram-lak_scikit", None)


def filterSinogram(sinogram, filter_name):
    """Filter along the detector axis, zero-padded to a power of two >= 2 nR (util/data.py:302-370)."""
    if filter_name is None or filter_name.lower() == "none":
        return sinogram
    if filter_name.lower() not in _SINO_FILTERS:
        raise ValueError("Unknown filter: %s" % filter_name)
    if sinogram.ndim not in (2, 3):
        raise Exception("The sinogram provided does not have compatible number of dimension (2 or 3).")
    pX = sinogram.shape[0]
    size = max(64, int(2 ** np.ceil(np.log2(2 * pX))))
    filt = _get_fourier_filter(size, filter_name)
    if sinogram.ndim == 2:
        img = np.pad(sinogram, ((0, size - pX), (0, 0)))
        return np.real(ifft(fft(img, axis=0) * filt, axis=0)[:pX, :])
    out = np.zeros(sinogram.shape, dtype=float)
    for z in range(sinogram.shape[2]):
        img = np.pad(sinogram[:, :, z], ((0, size - pX), (0, 0)))
        out[:, :, z] = np.real(ifft(fft(img, axis=0) * filt, axis=0)[:pX, :])
    return out


_FILTER_CACHE = {}


def _device_filter_half(size, filter_name, device):
    """The first size // 2 + 1 values of the real, even filter (the half spectrum of a real transform),
    float64 on the device, cached per (size, name, device)."""
    import torch

    key = (size, filter_name, str(device))
    if key not in _FILTER_CACHE:
        f = _get_fourier_filter(size, filter_name)[: size // 2 + 1, 0]
        _FILTER_CACHE[key] = torch.as_tensor(np.ascontiguousarray(f), device=device, dtype=torch.float64)
    return _FILTER_CACHE[key]


def filterSinogram_t(sino, filter_name, scale=1.0, lo=None, hi=None, out=None):
    """Device version of filterSinogram for a [nR, nA, nZ] (or [nR, nA]) torch tensor, followed by
    ``clip(scale * filtered, lo, hi)`` and returned as float32 (``out`` if given).

    The filter is real and even, so the reference's complex FFT of the zero-padded real columns times the
    filter, inverted and cropped to its real part, equals cuFFT's real-to-complex transform along the
    padded detector axis, the half spectrum times the filter's first size // 2 + 1 values
    (vam_spectrum_scale), the complex-to-real inverse and the crop; the crop, scale, clip and float32
    conversion are one pass (vam_filter_epilogue)."""
    import torch

    from .. import _lib

    if filter_name is None or filter_name.lower() == "none":
        x = sino.to(torch.float64)
    else:
        if filter_name.lower() not in _SINO_FILTERS:
            raise ValueError("Unknown filter: %s" % filter_name)
        pX = sino.shape[0]
        size = max(64, int(2 ** np.ceil(np.log2(2 * pX))))
        m = sino[0].numel()
        spec = torch.fft.rfft(sino.to(torch.float64).reshape(pX, m), n=size, dim=0).contiguous()
        filt = _device_filter_half(size, filter_name, sino.device)
        st = _lib.stream_ptr(torch.cuda.current_stream(sino.device))
        _lib.call("vam_spectrum_scale", _lib.ptr(spec), _lib.ptr(filt), spec.shape[0], m, st)
        x = torch.fft.irfft(spec, n=size, dim=0)
    if out is None:
        out = torch.empty(sino.shape, dtype=torch.float32, device=sino.device)
    pX, m = sino.shape[0], sino[0].numel()
    x = x.contiguous()
    _lib.call("vam_filter_epilogue", _lib.ptr(x), pX, m, float(scale), int(lo is not None),
              float(lo if lo is not None else 0.0), int(hi is not None), float(hi if hi is not None else 0.0),
              _lib.ptr(out), _lib.stream_ptr(torch.cuda.current_stream(sino.device)))
    return out


def discretize(x, bit_depth, range, output_dtype=float):
    """Quantise to 2**bit_depth levels of np.linspace(range) (util/data.py:495-523)."""
    assert len(range) == 2, "range argument should have 2 elements [min,max]"
    bins = np.linspace(range[0], range[1], 2 ** bit_depth, endpoint=True)
    return bins[np.digitize(x, bins=bins) - 1].astype(output_dtype)


def discretize_t(x, bit_depth, lo, hi):
    """Device version of discretize for a torch tensor (lo / hi python or 0-d tensors)."""
    import torch

    n = 2 ** bit_depth
    t = torch.linspace(0.0, 1.0, n, device=x.device, dtype=torch.float64)
    lo = torch.as_tensor(lo, device=x.device, dtype=torch.float64)
    hi = torch.as_tensor(hi, device=x.device, dtype=torch.float64)
    bins = lo + (hi - lo) * t
    idx = torch.bucketize(x.to(torch.float64), bins, right=True) - 1
    idx = idx % n  # np.digitize below the first bin gives -1 -> last bin (numpy wraps)
    return bins[idx].to(x.dtype)
