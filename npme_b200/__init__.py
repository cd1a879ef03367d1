"""npme_b200: B200-native (sm_100a) NPME potential evaluation.

The compute path is the CUDA library ``libnpme_gpu.so`` built from
``npme_b200/csrc`` (``python -m npme_b200.build``); this package is a thin
ctypes binding of its C ABI (``include/npme_gpu.h``).  There is no CPU
fallback: importing works without a GPU, but creating a solver raises when
the library is missing or no CUDA device is usable.
"""
from .api import (NPMEError, Params, Solver, lib_path, load_library,  # noqa: F401
                  PREC_FP32, PREC_FP64)
from .workloads import Workload, CONFIGS  # noqa: F401
