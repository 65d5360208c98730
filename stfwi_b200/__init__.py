"""B200-native (sm_100a) elastic velocity-strain modelling, adjoint and
gradients: a drop-in for the hot path of the reference's ``fwi`` package."""
from .solver import Solver  # noqa: F401
