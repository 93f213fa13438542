"""Algebraic (sparse-matrix) propagation on the B200.

``PyTorchAlgebraicPropagator`` mirrors the reference's class of the same name
(vamtoolbox/projector/pyTorchAlgebraicPropagation.py:13-181): it loads a
propagation matrix (rows = sinogram elements, columns = voxels) from the
``.npz`` (SciPy) or ``.pt`` (PyTorch) file named by
``proj_geo.loading_path_for_matrix``, or takes one directly (``matrix=``, e.g.
the output of ``PyTorchRayTracingPropagator.buildPropagationMatrix``), and
applies it with the reference's z tiling: a matrix built for one z layer is
applied to every layer of a volume whose voxel count is a multiple of its
column count.  Forward and backward run the CSR kernel ``vam_csr_spmm`` on
the matrix and on its transpose (built once by a stable sort, so both are
deterministic).  ``AlgebraicPropagator`` (the reference's SciPy CPU class,
vamtoolbox/projector/algebraicPropagation.py) is the same class here.
"""
from __future__ import annotations

import logging
import os

import numpy as np
import torch

from .. import _lib


def _to_coo(matrix):
    """(rows int64, cols int64, vals float32, shape) on the CPU from a scipy sparse matrix or torch sparse tensor."""
    if isinstance(matrix, torch.Tensor):
        m = matrix.to_sparse_coo().coalesce().cpu() if matrix.layout != torch.sparse_coo else matrix.coalesce().cpu()
        idx = m.indices()
        return idx[0].to(torch.int64), idx[1].to(torch.int64), m.values().to(torch.float32), tuple(m.shape)
    import scipy.sparse

    m = scipy.sparse.coo_matrix(matrix)
    m.sum_duplicates()
    return (torch.as_tensor(m.row, dtype=torch.int64), torch.as_tensor(m.col, dtype=torch.int64),
            torch.as_tensor(m.data, dtype=torch.float32), tuple(m.shape))


def _csr(rows, cols, vals, n_rows, device):
    """CSR arrays (row_ptr int64, cols int32, vals float32) on device from COO sorted by (row, col)."""
    order = torch.argsort(rows * (int(cols.max()) + 1 if cols.numel() else 1) + cols, stable=True)
    rows, cols, vals = rows[order], cols[order], vals[order]
    row_ptr = torch.zeros(n_rows + 1, dtype=torch.int64)
    if rows.numel():
        row_ptr[1:] = torch.cumsum(torch.bincount(rows, minlength=n_rows), 0)
    return row_ptr.to(device), cols.to(torch.int32).to(device), vals.to(device)


class PyTorchAlgebraicPropagator:
    """P in P f = g as a sparse matrix (pyTorchAlgebraicPropagation.py:13-181)."""

    def __init__(self, target_geo, proj_geo, output_torch_tensor=False, dtype=torch.float32, matrix=None,
                 device=None):
        self.logger = logging.getLogger(__name__)
        if not torch.cuda.is_available():
            raise RuntimeError("vamtoolbox_b200 propagators need a CUDA device (no CPU fallback)")
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.output_torch_tensor = output_torch_tensor
        self.dtype = dtype
        if matrix is None:
            file_path = proj_geo.loading_path_for_matrix
            ext = os.path.splitext(str(file_path))[-1].lower()
            if ext == ".npz":
                import scipy.sparse

                try:
                    matrix = scipy.sparse.load_npz(file_path)
                except OSError:
                    raise Exception(f'Sparse matrix file at "{file_path}" does not exist or cannot be read.')
            elif ext == ".pt":
                try:
                    matrix = torch.load(file_path, map_location="cpu")
                except OSError:
                    raise Exception(f'PyTorch tensor file at "{file_path}" does not exist or cannot be read.')
            else:
                raise Exception("Invalid file format. Supported formats: .npz (SciPy) or .pt (PyTorch)")
        rows, cols, vals, shape = _to_coo(matrix)
        self.n_row_internal, self.n_col_internal = shape
        self.internal_matrix_shape = shape
        self._A = _csr(rows, cols, vals, self.n_row_internal, self.device)
        self._AT = _csr(cols, rows, vals, self.n_col_internal, self.device)
        self.n_col_eff = int(np.asarray(target_geo.array).size)
        if self.n_col_eff % self.n_col_internal != 0:
            raise Exception(f"The imported sparse matrix has {self.n_col_internal} columns, and it cannot match or be "
                            f"tiled to match the total number of voxels ({self.n_col_eff}) in the real space target.")
        self.z_tiling = self.n_col_eff // self.n_col_internal
        self.n_row_eff = self.n_row_internal * self.z_tiling
        self.shape = (self.n_row_eff, self.n_col_eff)

    def _apply(self, csr, n_out_rows, x):
        row_ptr, cols, vals = csr
        x = torch.as_tensor(x, device=self.device).to(torch.float32).reshape(-1, self.z_tiling).contiguous()
        y = torch.empty((n_out_rows, self.z_tiling), dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.call("vam_csr_spmm", n_out_rows, _lib.ptr(row_ptr), _lib.ptr(cols), _lib.ptr(vals), _lib.ptr(x),
                      self.z_tiling, _lib.ptr(y), _lib.stream_ptr(torch.cuda.current_stream(self.device)))
        y = y.flatten().to(self.dtype)
        return y if self.output_torch_tensor else y.cpu().numpy()

    def _spmm_into(self, csr, n_out_rows, x, out):
        row_ptr, cols, vals = csr
        _lib.call("vam_csr_spmm", n_out_rows, _lib.ptr(row_ptr), _lib.ptr(cols), _lib.ptr(vals), _lib.ptr(x),
                  self.z_tiling, _lib.ptr(out), _lib.stream_ptr(torch.cuda.current_stream(self.device)))
        return out

    def forward_t(self, x, out):
        """b = P x into ``out`` on the current stream: x and out contiguous float32 tensors on the device
        with n_col_eff and n_row_eff elements.  Allocates nothing (the fused BCLP engine captures it)."""
        return self._spmm_into(self._A, self.n_row_internal, x, out)

    def backward_t(self, b, out):
        """x = P^T b into ``out`` on the current stream (as forward_t)."""
        return self._spmm_into(self._AT, self.n_col_internal, b, out)

    def forward(self, x):
        """b = P x, x of n_col_eff voxels (z tiled), b of n_row_eff elements (pyTorchAlgebraicPropagation.py:146-163)."""
        return self._apply(self._A, self.n_row_internal, x)

    def backward(self, b):
        """x = P^T b (pyTorchAlgebraicPropagation.py:165-181)."""
        return self._apply(self._AT, self.n_col_internal, b)


AlgebraicPropagator = PyTorchAlgebraicPropagator
