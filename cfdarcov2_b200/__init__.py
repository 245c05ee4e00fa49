"""B200-native finite-volume time step for the cfdARCO operator API.

The product is libcfdb.so (C ABI in include/cfdb.h, CUDA kernels for
sm_100a under csrc/) and the drop-in C++ facade (include/cfdb/).  This Python
package only binds the C ABI for tests and benchmarks.  It has no other
implementation: when libcfdb.so is present it is loaded at import, and when
it is not (a fresh checkout, before ``python -m cfdarcov2_b200.build``, which
itself imports this package) every call into the library raises ImportError.
"""
import os as _os

from . import capi  # noqa: F401
from .capi import F32, F64, FUSED, PLAIN, CfdbError, lib  # noqa: F401

if _os.path.exists(capi.LIB_PATH):
    lib()  # load (and bind) the CUDA library now; a broken build fails here

from .api import (Batch, Context, Euler, Mesh, load_state, revolve_plan, save_state,  # noqa: E402,F401
                  write_mesh_json, write_vti)
