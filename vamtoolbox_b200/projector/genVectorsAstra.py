"""vamtoolbox.projector.genVectorsAstra: the ASTRA parallel3d_vec rows of an inclined (laminography)
geometry (vamtoolbox/projector/genVectorsAstra.py:4-53), built in projector/Projector3DParallelCUDA.py."""
from .Projector3DParallelCUDA import genVectorsAstra

__all__ = ["genVectorsAstra"]
