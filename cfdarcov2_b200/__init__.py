"""B200-native finite-volume time step for the cfdARCO operator API.

The product is libcfdb.so (C ABI in include/cfdb.h, CUDA kernels for
sm_100a under csrc/) and the drop-in C++ facade (include/cfdb/).  This Python
package only binds the C ABI for tests and benchmarks; importing it fails if
the library has not been built (``python -m cfdarcov2_b200.build``).
"""
from . import capi  # noqa: F401
from .capi import F32, F64, FUSED, PLAIN, CfdbError, lib  # noqa: F401

lib()  # fail loudly at import time when the CUDA library is missing

from .api import Batch, Context, Euler, Mesh, revolve_plan, write_mesh_json, write_vti  # noqa: E402,F401
