"""Projector frames from a sinogram: the reference's ``vamtoolbox.imagesequence``.

Mirrors vamtoolbox/imagesequence.py: ImageConfig (:14-82), ImageSeq (:85-284),
loadImageSeq (:287-293), the insertion helpers _insertImage /
_arrayInsertImage (:296-355) and the plane transforms _invertU / _invertV /
_scaleSize / _scaleIntensity / _truncateIntensity / _rotate (:358-401).

The whole chain runs on the GPU through libvamcore:
  flips and rotation      vam_sino_rotate   (flips alone are folded into the
                                             frame tables, no pass of their own)
  resize                  vam_sino_resize
  percentile              vam_select_pair   (the two sorted elements numpy blends)
  normalise, scale, truncate, cast, insert into N_v x N_u uint8 frames
                          vam_imageseq_frames
The host computes only what is O(frame edge): the rotation matrix, the frame
placement tables and numpy's blend of the two order statistics, each in the
dtypes numpy uses, so the frames are the reference's frames.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import ArgumentError

import numpy as np

from . import _lib
from .geometry import Sinogram


class ImageConfig:
    """Placement and intensity options of the frames (imagesequence.py:14-82).

    ``image_dims`` = (image width N_u, image height N_v), both multiples of 4.
    Keywords: rotate_angle (degrees), u_offset, v_offset, invert_u, invert_v,
    array_num, array_offset, normalization_percentile, intensity_scale,
    bit_depth, size_scale -- the reference's names and defaults.
    """

    def __init__(self, image_dims, **kwargs):
        self.N_u, self.N_v = image_dims
        if self.N_u % 4 != 0 or self.N_v % 4 != 0:
            raise Exception("Image dimensions should be divisible by 4.")
        self.rotate_angle = kwargs.get("rotate_angle", 0.0)
        self.u_offset = kwargs.get("u_offset", 0)
        self.v_offset = kwargs.get("v_offset", 0)
        self.invert_u = kwargs.get("invert_u", False)
        self.invert_v = kwargs.get("invert_v", False)
        self.array_num = kwargs.get("array_num", 1)
        self.array_offset = kwargs.get("array_offset", 0)
        self.normalization_percentile = kwargs.get("normalization_percentile", None)
        self.intensity_scale = kwargs.get("intensity_scale", 1.0)
        self.bit_depth = kwargs.get("bit_depth", 8)
        self.size_scale = kwargs.get("size_scale", 1.0)


# --------------------------------------------------------------------------
# host-side pieces (O(frame edge) work, in numpy's own dtypes)
# --------------------------------------------------------------------------

def rotation_plan(n_r, n_z, angle_deg):
    """Output plane shape and affine map of ndimage.rotate(..., axes=(0, 2),
    reshape=True) for an (n_r, n_z) plane (imagesequence.py:396-401).

    Returns ((o_r, o_z), [m00, m01, m10, m11, off0, off1]): output (o0, o1)
    samples the input at (m00*o0 + off0 + m01*o1, m10*o0 + off1 + m11*o1).
    The degree-exact cosine / sine are scipy.special's cosdg / sindg, the
    functions ndimage.rotate itself calls.
    """
    from scipy import special

    c, s = special.cosdg(angle_deg), special.sindg(angle_deg)
    rot = np.array([[c, s], [-s, c]])
    in_plane = np.asarray([n_r, n_z])
    iy, ix = in_plane
    bounds = rot @ [[0, 0, iy, iy], [0, ix, 0, ix]]
    out_plane = (np.ptp(bounds, axis=1) + 0.5).astype(int)
    offset = (in_plane - 1) / 2 - rot @ ((out_plane - 1) / 2)
    affine = [rot[0, 0], rot[0, 1], rot[1, 0], rot[1, 1], offset[0], offset[1]]
    return (int(out_plane[0]), int(out_plane[1])), [float(v) for v in affine]


def copy_offsets(cfg):
    """Per-copy extra v offsets passed to _insertImage (imagesequence.py:157-173, 329-355).

    A single image is inserted with v_offset 0; arrayed copies use the
    reference's alternating sequence, which already contains cfg.v_offset
    (so _insertImage subtracts it a second time, as the reference does).
    array_num <= 0 inserts nothing.
    """
    if cfg.array_num == 1:
        return [0]
    offsets = []
    for k in range(cfg.array_num):
        if cfg.array_num % 2 == 0:
            array_dir = int(np.ceil((k + 1) / 2) * (-1) ** k)            # 1, -1, 2, -2, ...
            offsets.append(int(cfg.array_offset * array_dir / 2 + cfg.v_offset))
        else:
            array_dir = int(0 + np.ceil(k / 2) * (-1) ** (k + 1))        # 0, 1, -1, 2, -2, ...
            offsets.append(int(cfg.array_offset * array_dir + cfg.v_offset))
    return offsets


def insert_boxes(cfg, s_u, s_v):
    """Frame rectangles (u1, u2, v1, v2), one per inserted copy in insertion
    order, of an s_v x s_u image (_insertImage, imagesequence.py:303-326).

    Raises the reference's exceptions for an image that does not fit, and
    numpy's broadcast ValueError where the truncated bounds span fewer pixels
    than the image.
    """
    boxes = []
    for v_off in copy_offsets(cfg):
        u1 = int(cfg.N_u / 2 - cfg.u_offset - s_u / 2)
        u2 = int(cfg.N_u / 2 - cfg.u_offset + s_u / 2)
        v1 = int(cfg.N_v / 2 - cfg.v_offset - v_off - s_v / 2)
        v2 = int(cfg.N_v / 2 - cfg.v_offset - v_off + s_v / 2)
        if u1 < 0 or u2 > cfg.N_u:
            raise Exception(
                "Image could not be inserted because it is either too large in the u-dimension or the offset "
                "causes it to extend out of the input screen size")
        if v1 < 0 or v2 > cfg.N_v:
            raise Exception(
                "Image could not be inserted because it is either too large in the v-dimension or the offset "
                "causes it to extend out of the input screen size")
        if (v2 - v1, u2 - u1) != (s_v, s_u):
            raise ValueError(f"could not broadcast input array from shape ({s_v},{s_u}) into shape "
                             f"({v2 - v1},{u2 - u1})")
        boxes.append((u1, u2, v1, v2))
    return boxes


def placement_tables(cfg, s_u, s_v, n_r, n_z, flip_r=False, flip_z=False):
    """Frame column -> sinogram row and frame row -> sinogram z tables.

    The image of angle j is sino[:, j, :].T (s_v = z extent rows, s_u = r
    extent columns), inserted by _insertImage once per copy
    (:func:`insert_boxes`); a later copy overwrites an earlier one.  Flips not
    applied by a plane transform are folded in here (_invertU / _invertV,
    imagesequence.py:358-365).  -1 marks blank pixels.
    """
    src_col = np.full(cfg.N_u, -1, dtype=np.int32)
    src_row = np.full(cfg.N_v, -1, dtype=np.int32)
    for u1, u2, v1, v2 in insert_boxes(cfg, s_u, s_v):
        cols = np.arange(s_u, dtype=np.int32)
        rows = np.arange(s_v, dtype=np.int32)
        src_col[u1:u2] = (n_r - 1 - cols) if flip_r else cols
        src_row[v1:v2] = (n_z - 1 - rows) if flip_z else rows
    return src_col, src_row


def table_box(src_col, src_row):
    """Bounding box (v0, v1, u0, u1) of the non-blank table entries."""
    rows = np.flatnonzero(src_row >= 0)
    cols = np.flatnonzero(src_col >= 0)
    if rows.size == 0 or cols.size == 0:
        return 0, 0, 0, 0
    return int(rows[0]), int(rows[-1]) + 1, int(cols[0]), int(cols[-1]) + 1


def percentile_ranks(n, p, dtype):
    """Ranks and weight numpy's linear percentile uses (numpy percentile /
    _quantile, method 'linear', as called at imagesequence.py:129-131).

    q = p / dtype(100) and the virtual index (n - 1) * q are computed in the
    dtypes numpy gives them (float32 for a float32 array and a Python p);
    returns (k0, k1, gamma) with k1 in {k0, k0 + 1}.
    """
    q = np.true_divide(p, dtype.type(100))
    if not (np.all(0 <= q) and np.all(q <= 1)):
        raise ValueError("Percentiles must be in the range [0, 100]")
    vi = np.asanyarray((n - 1) * q)
    prev = np.asanyarray(np.floor(vi))
    if np.isnan(vi) or vi >= n - 1:
        k0 = k1 = n - 1
    elif vi < 0:
        k0 = k1 = 0
    else:
        k0 = int(prev)
        k1 = k0 + 1
    gamma = np.asanyarray(vi - prev, dtype=vi.dtype)
    return k0, k1, gamma


def blend(a, b, t):
    """numpy's percentile interpolation between sorted neighbours a <= b:
    a + (b - a) * t, or b - (b - a) * (1 - t) when t >= 0.5, in numpy's
    result dtype; returns a numpy scalar."""
    a = np.asanyarray(a)
    b = np.asanyarray(b)
    diff = np.subtract(b, a)
    out = np.asanyarray(np.add(a, diff * t))
    np.subtract(b, diff * (1 - t), out=out, where=t >= 0.5, casting="unsafe", dtype=type(out.dtype))
    return out[()]


def _output_dtype(bit_depth):
    if bit_depth <= 8:
        return np.uint8
    if bit_depth <= 16:
        return np.uint16
    if bit_depth <= 32:
        return np.uint32
    raise ValueError("Bit depth higher than 32-bit is not supported.")


def _dtype_code(dt):
    dt = np.dtype(dt)
    if dt == np.float32:
        return _lib.DTYPE_F32
    if dt == np.float64:
        return _lib.DTYPE_F64
    raise TypeError(f"sinogram dtype {dt} is not supported (float32 or float64)")


def _torch_dtype(dt):
    import torch

    return torch.float64 if np.dtype(dt) == np.float64 else torch.float32


def _sinogram_array(sinogram):
    if isinstance(sinogram, Sinogram):
        return sinogram.array
    try:
        import torch

        if isinstance(sinogram, torch.Tensor):
            return sinogram
    except ImportError:  # pragma: no cover
        pass
    if isinstance(sinogram, np.ndarray):
        return sinogram
    raise ArgumentError("sinogram not specified.")


class _Prepared:
    """The sinogram after the plane transforms, on the device, with the
    quantiser parameters of the frame kernel (everything but the tables)."""


def _prepare(sinogram, cfg, device=None, stream=None):
    import torch

    arr = _sinogram_array(sinogram)
    if isinstance(arr, torch.Tensor):
        dev = arr.device if arr.is_cuda else torch.device("cuda", torch.cuda.current_device()
                                                          if device is None else device)
        np_dtype = np.float64 if arr.dtype == torch.float64 else (np.float32 if arr.dtype == torch.float32 else None)
        if np_dtype is None:
            raise TypeError(f"sinogram dtype {arr.dtype} is not supported (float32 or float64)")
        cur = arr.to(dev).contiguous()
    else:
        arr = np.asarray(arr)
        if arr.dtype not in (np.float32, np.float64):
            raise TypeError(f"sinogram dtype {arr.dtype} is not supported (float32 or float64)")
        np_dtype = arr.dtype.type
        dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        cur = torch.from_numpy(np.ascontiguousarray(arr)).to(dev)
    if cur.dim() != 3:
        raise IndexError(f"too many indices for array: array is {cur.dim()}-dimensional, but 3 were indexed")
    _lib.load()
    P = _Prepared()
    P.dev = dev
    with torch.cuda.device(dev):
        st = _lib.stream_ptr(stream)
        cur_dt = np.dtype(np_dtype)
        flip_r, flip_z = bool(cfg.invert_u), bool(cfg.invert_v)
        n_r, n_a, n_z = cur.shape
        if cfg.rotate_angle != 0.0:
            (o_r, o_z), affine = rotation_plan(n_r, n_z, cfg.rotate_angle)
            out = torch.empty((o_r, n_a, o_z), dtype=cur.dtype, device=dev)
            aff = (_lib._c_d * 6)(*affine)
            _lib.call("vam_sino_rotate", _lib.ptr(cur), _dtype_code(cur_dt), n_r, n_a, n_z, int(flip_r),
                      int(flip_z), aff, _lib.ptr(out), o_r, o_z, st)
            cur, flip_r, flip_z = out, False, False
            n_r, n_z = o_r, o_z
        if cfg.size_scale != 1.0:
            o_r, o_z = int(n_r * cfg.size_scale), int(n_z * cfg.size_scale)
            if o_r <= 0 or o_z <= 0:
                raise ValueError(f"size_scale {cfg.size_scale} leaves an empty {o_r} x {o_z} plane")
            out = torch.empty((o_r, n_a, o_z), dtype=torch.float64, device=dev)
            _lib.call("vam_sino_resize", _lib.ptr(cur), _dtype_code(cur_dt), n_r, n_a, n_z, int(flip_r),
                      int(flip_z), _lib.ptr(out), o_r, o_z, st)
            cur, flip_r, flip_z, cur_dt = out, False, False, np.dtype(np.float64)
            n_r, n_z = o_r, o_z

        prm = _lib.FrameParams()
        _output_dtype(cfg.bit_depth)
        if not 0 <= cfg.bit_depth <= 32:
            raise ValueError(f"bit_depth {cfg.bit_depth} is outside 0..32")
        prm.bit_depth = int(cfg.bit_depth)
        stage_dt = cur_dt
        if cfg.normalization_percentile is not None:
            n = cur.numel()
            k0, k1, gamma = percentile_ranks(n, cfg.normalization_percentile, cur_dt)
            pair = torch.empty(2, dtype=cur.dtype, device=dev)
            wbytes = _lib.load().vam_select_workspace_bytes()
            work = torch.empty(wbytes, dtype=torch.uint8, device=dev)
            _lib.call("vam_select_pair", _lib.ptr(cur), _dtype_code(cur_dt), n, k0, k1, _lib.ptr(pair),
                      _lib.ptr(work), wbytes, st)
            lo, hi = pair.cpu().numpy()
            norm = blend(lo, hi, gamma)
            stage_dt = np.result_type(np.empty(0, stage_dt), norm)
            prm.has_norm = 1
            prm.norm_value = float(norm)
            prm.norm_dtype = _dtype_code(np.asarray(norm).dtype)
        if cfg.intensity_scale != 1.0:
            scaled_dt = np.result_type(np.empty(0, stage_dt), cfg.intensity_scale)
            prm.has_scale = 1
            prm.intensity_scale = float(cfg.intensity_scale)
            prm.scale_is_f64 = int(scaled_dt == np.float64)
    P.cur, P.cur_dt, P.shape, P.flips, P.prm, P.stream = cur, cur_dt, (n_r, n_a, n_z), (flip_r, flip_z), prm, st
    return P


def _launch_frames(P, src_col, src_row, n_u, n_v, box, out):
    import torch

    prm = P.prm
    prm.n_u, prm.n_v = int(n_u), int(n_v)
    prm.box_v0, prm.box_v1, prm.box_u0, prm.box_u1 = box
    with torch.cuda.device(P.dev):
        col_d = torch.from_numpy(src_col).to(P.dev)
        row_d = torch.from_numpy(src_row).to(P.dev)
        prm.src_col_dev = col_d.data_ptr()
        prm.src_row_dev = row_d.data_ptr()
        n_r, n_a, n_z = P.shape
        if n_a > 0:
            _lib.call("vam_imageseq_frames", _lib.ptr(P.cur), _dtype_code(P.cur_dt), n_r, n_a, n_z,
                      ctypes.byref(prm), _lib.ptr(out), P.stream)
    return out


def device_frames(sinogram, cfg, device=None, stream=None):
    """Run the frame pipeline on the GPU; returns the [nA][N_v][N_u] uint8 frames on the device.

    ``sinogram``: numpy array, torch tensor (any device) or Sinogram, shape
    [nR][nA][nZ], float32 or float64.
    """
    import torch

    P = _prepare(sinogram, cfg, device, stream)
    n_r, n_a, n_z = P.shape
    src_col, src_row = placement_tables(cfg, n_r, n_z, n_r, n_z, *P.flips)
    frames = torch.empty((n_a, cfg.N_v, cfg.N_u), dtype=torch.uint8, device=P.dev)
    return _launch_frames(P, src_col, src_row, cfg.N_u, cfg.N_v, table_box(src_col, src_row), frames)


class ImageSeq:
    """Sinogram converted to projector frames (imagesequence.py:85-284).

    The frames are built on the GPU (:func:`device_frames`).  ``images`` is
    the reference's list of N_v x N_u uint8 arrays, one per angle (views of
    one page-locked [nA][N_v][N_u] host array).  ``keep_device_frames=True``
    also keeps the device copy as ``frames_device``, e.g. for a display
    pipeline; ``host_images=False`` skips the host copy (``images`` is None).
    """

    def __init__(self, image_config, sinogram, *, device=None, keep_device_frames=False, host_images=True):
        import torch

        self.file_extension = ".imgseq"
        self.image_config = image_config
        self.frames_device = None
        self.images = None
        frames = device_frames(sinogram, image_config, device=device)
        if keep_device_frames:
            self.frames_device = frames
        if host_images:
            # one DMA into page-locked memory (torch's host caching allocator
            # hands the block back for reuse once these images are released)
            host = torch.empty(frames.shape, dtype=torch.uint8, pin_memory=True)
            host.copy_(frames)
            arr = host.numpy()
            self.images = [arr[j] for j in range(arr.shape[0])]

    def __getstate__(self):
        d = dict(self.__dict__)
        d["frames_device"] = None
        if d.get("images") is not None:
            d["images"] = [np.array(im) for im in d["images"]]
        return d

    def __setstate__(self, d):
        self.__dict__ = d

    def save(self, name: str):
        """Save as 'name.imgseq' (dill pickle, imagesequence.py:183-187)."""
        import dill

        with open(name + self.file_extension, "wb") as fh:
            dill.dump(self, fh)

    def preview(self):
        """The reference previews through its pyglet DLP player (vamtoolbox/dlp/players.py), a windowing
        stack that is not part of this package: like ``show()`` on volumes, this logs that nothing is shown
        and returns, so a script runs to the end headless (the frames are ``self.images``; saveAsImages /
        saveAsVideo write them)."""
        import logging

        logging.getLogger(__name__).warning("ImageSeq.preview(): no display in this package; see .images")

    def saveAsVideo(self, save_path, rot_vel, num_loops=1, mode="conventional", angle_increment_per_image=None,
                    preview=False):
        """Write the frames as a video with OpenCV (imagesequence.py:195-270)."""
        import cv2

        if self.images is None:
            raise Exception("Problem encountered creating images in ImageSeq initialization")
        if preview:
            raise NotImplementedError("video preview needs a display window, which this package does not provide")
        if mode == "conventional":
            assert angle_increment_per_image is None, (
                "angle_increment_per_image must be None in conventional mode because it is derived from number "
                "of images in sinogram")
            angle_increment_per_image = 360 / len(self.images)
            num_total_images = int(np.round(360.0 / angle_increment_per_image * num_loops))
        elif mode == "prescribed":
            assert angle_increment_per_image is not None, (
                "angle_increment_per_image must be None in conventional mode because it is derived from number "
                "of images in sinogram")
            num_total_images = int(len(self.images) * num_loops)
        else:
            raise Exception('mode argument is not valid. Either "conventional" or "prescribed"')
        fps = 1 / (angle_increment_per_image / rot_vel)
        out = cv2.VideoWriter(save_path, cv2.VideoWriter.fourcc(*"avc1"), fps,
                              (int(self.image_config.N_u), int(self.image_config.N_v)), isColor=False)
        for k in range(num_total_images):
            out.write(self.images[k % len(self.images)])
        out.release()

    def saveAsImages(self, save_dir, image_prefix="image", image_type=".png"):
        """One image file per frame, name prefix + 4-digit index (imagesequence.py:272-284)."""
        from PIL import Image

        for k, image in enumerate(self.images):
            path = os.path.join(save_dir, image_prefix + str(k).zfill(4) + image_type)
            Image.fromarray(image).save(path, subsampling=0, quality=100)


def loadImageSeq(file_name: str):
    """Load an ImageSeq saved with ImageSeq.save (imagesequence.py:287-293)."""
    import dill

    with open(file_name, "rb") as fh:
        return dill.loads(fh.read())
