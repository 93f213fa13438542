"""Array helpers (vamtoolbox.util counterpart)."""
from . import build_sparse_matrix, data, matlab, thresholding, timing
