"""vamtoolbox_b200: the tomographic projection hot path of VAMToolbox on B200 (sm_100a).

Drop-in modules with the reference's names: ``geometry``, ``projectorconstructor``,
``optimize``, ``medium``, ``response``, ``metrics``, ``util.data``.  The
projection kernels live in ``libvamcore.so`` (include/vam.h); build it with
``python -m vamtoolbox_b200.csrc.build``.
"""
__version__ = "0.1.0"

from . import util
from . import geometry
from . import medium
