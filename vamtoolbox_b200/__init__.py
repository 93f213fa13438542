"""vamtoolbox_b200: the tomographic projection hot path of VAMToolbox on B200 (sm_100a).

Drop-in modules with the reference's names, imported with the package as the reference's are:
``geometry``, ``projectorconstructor``, ``optimize``, ``optimizer``, ``projector``, ``medium``,
``response``, ``metrics``, ``imagesequence``, ``resources``, ``util``.  The
projection kernels live in ``libvamcore.so`` (include/vam.h); build it with
``python -m vamtoolbox_b200.csrc.build``.
"""
__version__ = "0.1.0"

from . import util
from . import geometry
from . import medium
from . import response
from . import metrics
from . import resources
from . import projector
from . import projectorconstructor
from . import optimizer
from . import optimize
from . import imagesequence
