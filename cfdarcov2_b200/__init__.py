"""B200-native finite-volume time step for the cfdARCO operator API.

The product is libcfdb.so (C ABI in include/cfdb.h, CUDA kernels for
sm_100a under csrc/) and the drop-in C++ facade (include/cfdb/).  This Python
package only binds the C ABI for tests and benchmarks.  It has no other
implementation: libcfdb.so is loaded by the first call into it (creating a
``Context`` or calling ``lib()``), and when it is not built that first call
raises ImportError.  Importing the package, or its numpy-only ``workloads``
module, maps no native code, so a CPU-only process (the timed CPU
restatement) can build the same synthetic inputs without loading the CUDA
library.
"""
from . import capi  # noqa: F401
from .api import (Batch, Context, Euler, Mesh, load_state, revolve_plan, save_state,  # noqa: F401
                  write_mesh_json, write_vti)
from .capi import F32, F64, FUSED, PLAIN, CfdbError, lib  # noqa: F401
