"""B200-native VUMPS / IDMRG / TDVP inner loop with the InfiniteMPSAlgorithms API.

The compute path is the sm_100a library ``libimps_b200.so`` (C ABI in
``include/imps_b200.h``); this package is the host-side mirror of the
reference's Julia API.  Importing the package does not touch the GPU; the
first call that needs the device loads the library and raises if it (or a
CUDA device) is missing -- there is no CPU fallback.
"""
from .api import *  # noqa: F401,F403
from .api import __all__ as _api_all
from ._lib import (ImpsError, DimensionMismatch, ArgumentError, IMPS_PREC_FP64,  # noqa: F401
                   IMPS_PREC_SPLIT_I8, LIB_PATH)

__all__ = list(_api_all) + ["ImpsError", "DimensionMismatch", "ArgumentError", "IMPS_PREC_FP64",
                            "IMPS_PREC_SPLIT_I8", "LIB_PATH"]
