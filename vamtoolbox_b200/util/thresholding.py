"""vamtoolbox.util.thresholding (vamtoolbox/util/thresholding.py:5-6)."""
import numpy as np


def threshold(x, thresh):
    """Boolean array of x >= thresh."""
    return (np.asarray(x) >= thresh).astype(np.bool_)
