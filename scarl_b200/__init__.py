"""scarl_b200: the ScaRL random-field path on NVIDIA B200 (sm_100a).

The CUDA library libscarl_b200.so (built in-tree by scarl_b200.build) carries
every kernel and the C ABI of include/scarl.h; this package is its Python
front end.  Importing it without the built library raises ImportError.
"""
from ._lib import (CM_EXPONENTIAL, CM_GAUSSIAN, CM_VON_KARMAN, F32, F64, FOM_GAUSSIAN,
                   FOM_LOGNORMAL, GEN_DCT, GEN_PADDED, GEN_SHINO, PAD_AUTO, PAD_FULL, PAD_LEARNED,
                   PAD_SMOOTH,
                   SPLIT_BF16, SPLIT_BF16_X, ScarlError,
                   lib)
from .api import *  # noqa: F401,F403

lib()  # fail loudly now, not at the first call
