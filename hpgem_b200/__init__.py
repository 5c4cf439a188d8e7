"""hpgem_b200: B200-native explicit DG time stepping for hpGEM's
HpgemAPISimplified path (linear advection, linear acoustic wave) and its
stored-matrix variant HpgemAPILinear.

The solver runs in the native library ``_lib/libhpgem_b200.so`` (C ABI in
include/hpgem_b200.h): CUDA kernels for sm_100a plus the C++ host set-up.
Build it with ``python -m hpgem_b200.build``.
"""
from ._native import NativeError, ProblemDesc, load  # noqa: F401
from .batch import Batch  # noqa: F401
from .server import Server  # noqa: F401
from .solver import (AcousticWave, Advection, Handle, HpgemAPILinear, HpgemAPISimplified,  # noqa: F401
                     structured_description)

__all__ = ["AcousticWave", "Advection", "Batch", "Handle", "Server", "HpgemAPILinear", "HpgemAPISimplified",
           "NativeError",
           "ProblemDesc", "load", "structured_description"]
