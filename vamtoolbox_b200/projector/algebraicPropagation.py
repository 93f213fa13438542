"""vamtoolbox.projector.algebraicPropagation: the reference's SciPy algebraic propagator
(vamtoolbox/projector/algebraicPropagation.py) is the device propagator here, the same class as
projector/pyTorchAlgebraicPropagation.py (CSR products on the GPU, the reference's z tiling)."""
from .pyTorchAlgebraicPropagation import AlgebraicPropagator, PyTorchAlgebraicPropagator

__all__ = ["AlgebraicPropagator", "PyTorchAlgebraicPropagator"]
