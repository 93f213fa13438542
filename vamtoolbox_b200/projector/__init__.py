"""Projectors of the B200 core (parallel beam and curved-ray tracer)."""
from . import Projector3DParallel
from . import pyTorchRayTrace
from .Projector3DParallel import Projector3DParallel as Projector3DParallelB200
