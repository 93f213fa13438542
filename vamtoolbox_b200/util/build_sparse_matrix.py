"""vamtoolbox.util.build_sparse_matrix (vamtoolbox/util/build_sparse_matrix.py:12-77): an explicit sparse
matrix of a projector, measured one sinogram element at a time."""
from __future__ import annotations

import logging
import time

import numpy as np
from scipy import sparse

from ..projectorconstructor import projectorconstructor

logger = logging.getLogger(__name__)


def buildMatrix(target_geo, proj_geo, sparse_format="csr", save_path=None, block_insert=False):
    """Row r of the matrix is the backprojection of the unit sinogram with a 1 at element r (the
    projector's shift-variant impulse response), flattened in C order; returned in ``sparse_format``
    (any scipy sparse format name) and saved to ``save_path`` (.npz) when given.  The rows are
    backprojected on the device and only their non-zeros are kept, so the matrix is assembled once
    in compressed form."""
    if block_insert:
        raise Exception("Block insertsion is not yet implemented.")
    A = projectorconstructor(target_geo, proj_geo)
    vol = np.zeros_like(target_geo.array)
    sino_shape = np.asarray(A.forward(vol)).shape
    n_row, n_col = int(np.prod(sino_shape)), vol.size
    logger.info("Building sparse matrix with %d rows and %d columns.", n_row, n_col)
    unit = np.zeros(n_row)
    rows, cols, vals = [], [], []
    t0 = time.perf_counter()
    for r in range(n_row):
        unit[r - 1] = 0.0
        unit[r] = 1.0
        col = np.asarray(A.backward(unit.reshape(sino_shape))).ravel()
        nz = np.flatnonzero(col)
        rows.append(np.full(nz.size, r, dtype=np.int64))
        cols.append(nz)
        vals.append(col[nz])
    logger.info("Rows measured in %.1f s.", time.perf_counter() - t0)
    P = sparse.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                          shape=(n_row, n_col)).asformat(sparse_format)
    if save_path is not None:
        sparse.save_npz(save_path, P)
    return P
