"""linearalgebra_b200 -- B200-native sparse hot path of miaodi/linearAlgebra.

CSR SpMV (segmented-sum and ALBUS forms), level-scheduled triangular
solves, IC(0)-PCG (FP64 and mixed precision) and adjoints, as hand-written
sm_100a CUDA kernels behind the C-ABI in include/la_b200.h, with host
preprocessing (level sets, RCM, IC(0)) bit-identical to the reference.
"""
from .api import *  # noqa: F401,F403
from .api import __all__ as _api_all
from ._lib import LAError, lib  # noqa: F401

__all__ = list(_api_all) + ["lib"]
