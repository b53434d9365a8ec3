"""B200-native dual-resolution Gaussian-process HMC sampler (the dualgpmf path of asw221/dualres).

Host code drives hand-written sm_100a CUDA kernels through the C ABI declared in
include/dualres_b200.h; this package is the Python mirror of that ABI.
"""
from .api import (DR_COV_RBF, DR_COV_RQ, DrError, HMCParameters, MultiResData, MultiResParameters, Server,  # noqa: F401
                  debug_dual_averaging, fit_model, kernel_launches, kriging_matrix, lib)

__version__ = "0.1.0"
