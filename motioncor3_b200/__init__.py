"""mc3-b200: B200-native motion correction of cryo-EM movies.

Python binding of libmc3 (include/mc3.h).  The work runs in the native
library (hand-written sm_100a kernels + C++ host code); this module only
marshals arguments.  There is no Python or CPU fallback: if libmc3.so is
missing the import of the native library raises.
"""
from .api import (  # noqa: F401
    MC3Error,
    MotionCor3,
    Params,
    Result,
    lib,
    lib_path,
)

__all__ = ["MC3Error", "MotionCor3", "Params", "Result", "lib", "lib_path"]
