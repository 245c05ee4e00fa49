"""ctypes binding of libcfdb.so (the C ABI declared in include/cfdb.h).

This module is plumbing for the tests, the smoke check and bench.py: it loads
the in-tree library, declares the prototypes and turns non-zero status codes
into ``CfdbError``.  It never falls back to anything: if the library is
missing, importing the package fails.
"""
from __future__ import annotations

import ctypes as C
import os
import re

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "_lib", "libcfdb.so")
HEADER_PATH = os.path.join(os.path.dirname(_PKG), "include", "cfdb.h")

OK, EINVAL, ENOMEM, ECUDA, ETIMEOUT, ENUMERIC, EUNSUPPORTED, EIO = range(8)
F32, F64 = 0, 1
PLAIN, FUSED = 0, 1
OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_RSUB, OP_RDIV = range(6)
GEOM_NORMAL, GEOM_NORMAL_ALT, GEOM_AREA, GEOM_ALPHA_D, GEOM_LEN_C2F, GEOM_VOLUME, GEOM_CENTER, GEOM_IS_BOUNDARY = range(8)
MESH_COMPAT_AREA = 1
RV_ADVANCE, RV_TAKESHOT, RV_RESTORE, RV_FIRSTURN, RV_YOUTURN = 1, 2, 3, 4, 5

_P = C.c_void_p
_I = C.c_int
_I32 = C.c_int32
_I64 = C.c_int64
_D = C.c_double
_PP = C.POINTER(C.c_void_p)
_PI64 = C.POINTER(C.c_int64)
_PD = C.POINTER(C.c_double)
_PI = C.POINTER(C.c_int)
_PI32 = C.POINTER(C.c_int32)


class Problem(C.Structure):
    """cfdb_problem: one member of a batched ensemble."""
    _fields_ = [("n", C.c_int32), ("kind", C.c_int32), ("param", C.c_double), ("dt", C.c_double),
                ("offset", C.c_int64)]


class GradientStats(C.Structure):
    """cfdb_gradient_stats."""
    _fields_ = [("forward_steps", C.c_int64), ("adjoint_steps", C.c_int64), ("snapshots_used", C.c_int32),
                ("reserved", C.c_int32), ("forward_ms", C.c_double), ("reverse_ms", C.c_double)]


class PlainGeometry(C.Structure):
    """cfdb_plain_geometry: device pointers of a mesh's FP32 face arrays."""
    _fields_ = [("ids", C.c_void_p), ("normal", C.c_void_p), ("normal_alt", C.c_void_p), ("area", C.c_void_p),
                ("alpha", C.c_void_p), ("len", C.c_void_p), ("volume", C.c_void_p), ("n", C.c_int64)]


class LatticeGeometry(C.Structure):
    """cfdb_lattice_geometry: per-slot FP32 constants of an exact lattice."""
    _fields_ = [("nx", C.c_int64), ("ny", C.c_int64), ("nz", C.c_int64), ("exact", C.c_int32),
                ("reserved", C.c_int32), ("normal", C.c_float * 18), ("normal_alt", C.c_float * 18),
                ("area", C.c_float * 6), ("alpha", C.c_float * 12), ("len", C.c_float * 12), ("volume", C.c_float)]


# name -> (restype, argtypes)
PROTOTYPES = {
    "cfdb_abi_version": (_I, []),
    "cfdb_ctx_create": (_I, [_I, _PP]),
    "cfdb_ctx_destroy": (_I, [_P]),
    "cfdb_last_error": (C.c_char_p, [_P]),
    "cfdb_ctx_set_stream": (_I, [_P, _P]),
    "cfdb_sync": (_I, [_P]),
    "cfdb_ctx_set_alloc_budget": (_I, [_P, _I64]),
    "cfdb_ctx_allocated_bytes": (_I, [_P, _PI64]),
    "cfdb_ctx_trim": (_I, [_P]),
    "cfdb_ctx_launch_count": (_I, [_P, _PI64]),
    "cfdb_ctx_set_wait_limit": (_I, [_P, _I64, _I32]),
    "cfdb_kernel_build": (_I, [_P, C.c_char_p, C.c_char_p, _PP]),
    "cfdb_kernel_build_many": (_I, [_P, _I, C.POINTER(C.c_char_p), C.POINTER(C.c_char_p), _PP]),
    "cfdb_kernel_launch": (_I, [_P, _I64, _I, _P]),
    "cfdb_kernel_destroy": (_I, [_P]),
    "cfdb_kernel_info": (_I, [_P, _PI, _PI64, _PI]),
    "cfdb_mesh_plain_geometry": (_I, [_P, _P]),
    "cfdb_mesh_lattice_geometry": (_I, [_P, _P]),
    "cfdb_write_vti": (_I, [C.c_char_p, C.c_char_p, _I64, _I64, _I64, _P]),
    "cfdb_write_mesh_json": (_I, [C.c_char_p, _I64, _I64, _I64, _D, _D, _D, _P]),
    "cfdb_state_save": (_I, [C.c_char_p, _I, _I64, _I64, _I64, _I32, _I64, _D, _P]),
    "cfdb_state_load": (_I, [C.c_char_p, _I, _I64, _I64, _I64, _I32, _PI64, _PD, _P]),
    "cfdb_alloc": (_I, [_P, _I64, _PP]),
    "cfdb_free": (_I, [_P, _P]),
    "cfdb_upload": (_I, [_P, _P, _P, _I64]),
    "cfdb_download": (_I, [_P, _P, _P, _I64]),
    "cfdb_upload_async": (_I, [_P, _P, _P, _I64]),
    "cfdb_download_async": (_I, [_P, _P, _P, _I64]),
    "cfdb_mesh_create_structured": (_I, [_P, _I64, _I64, _I64, _D, _D, _D, _PP]),
    "cfdb_mesh_create_from_vertices": (_I, [_P, _I64, _I64, _I64, _D, _D, _D, _P, _I, _PP]),
    "cfdb_mesh_destroy": (_I, [_P]),
    "cfdb_mesh_info": (_I, [_P, _PI64, _PD, _PI]),
    "cfdb_mesh_geometry": (_I, [_P, _I, _P]),
    "cfdb_mesh_ids": (_I, [_P, _P, _P]),
    "cfdb_op_grad": (_I, [_P, _P, _I, _P, _P, _I]),
    "cfdb_op_lapl": (_I, [_P, _P, _I, _P, _P, _I]),
    "cfdb_op_stab": (_I, [_P, _P, _I, _P, _P, _I]),
    "cfdb_op_binary": (_I, [_P, _I, _I, _P, _P, _P, _I64]),
    "cfdb_op_scalar": (_I, [_P, _I, _I, _P, _D, _P, _I64]),
    "cfdb_op_neg": (_I, [_P, _I, _P, _P, _I64]),
    "cfdb_op_fill": (_I, [_P, _I, _P, _D, _I64]),
    "cfdb_op_d1t": (_I, [_P, _I, _P, _P, _D, _P, _I64]),
    "cfdb_op_d2t": (_I, [_P, _I, _P, _P, _P, _D, _I, _P, _I64]),
    "cfdb_op_boundary_copy": (_I, [_P, _P, _I, _P, _P, _P]),
    "cfdb_op_boundary_set": (_I, [_P, _P, _I, _P, _P]),
    "cfdb_op_boundary_set_many": (_I, [_P, _P, _I, _I32, _P, _P]),
    "cfdb_cfl_dt": (_I, [_P, _P, _I, _D, _D, _P, _P, _P, _P, _P, _PD]),
    "cfdb_total_fp64": (_I, [_P, _P, _I, _P, _PD]),
    "cfdb_total_fp64_noalloc": (_I, [_I, _P, _P, _D, _I64, _P, _P]),
    "cfdb_heat_step": (_I, [_P, _P, _I, _I, _P, _P, _D, _D]),
    "cfdb_d2t_step": (_I, [_P, _P, _I, _P, _P, _P, _D, _P, _I32, _D, _I]),
    "cfdb_heat_step_fixed": (_I, [_P, _P, _I, _P, _P, _D, _D, _P]),
    "cfdb_wave_step": (_I, [_P, _P, _I, _I, _P, _P, _P, _D, _I, _D]),
    "cfdb_wave_dt": (_I, [_P, _P, _D, _D, _PD]),
    "cfdb_heat_run": (_I, [_P, _P, _I, _I, _P, _P, _D, _D, _I32, _I, _PI]),
    "cfdb_wave_run": (_I, [_P, _P, _I, _I, _P, _P, _P, _D, _I, _D, _I32, _I, _PI]),
    "cfdb_euler_create": (_I, [_P, _P, _I, _I, _D, _D, _D, _I64, _PP]),
    "cfdb_euler_destroy": (_I, [_P]),
    "cfdb_euler_begin": (_I, [_P, _P]),
    "cfdb_euler_step": (_I, [_P, _P, _P]),
    "cfdb_euler_status": (_I, [_P, _PD, _PI64, _PI]),
    "cfdb_euler_totals": (_I, [_P, _P, _I64, _PI64]),
    "cfdb_euler_run": (_I, [_P, _P, _P, _I64, _PI64, _PI]),
    "cfdb_batch_create": (_I, [_P, C.POINTER(Problem), _I32, _PI64, _PP]),
    "cfdb_batch_destroy": (_I, [_P]),
    "cfdb_batch_set_config": (_I, [_P, _I32, _I32, _I32]),
    "cfdb_batch_get_config": (_I, [_P, _PI32, _PI32, _PI32]),
    "cfdb_batch_set_staged": (_I, [_P, _I]),
    "cfdb_batch_tune": (_I, [_P, _P, _P, C.c_char_p]),
    "cfdb_batch_step": (_I, [_P, _P, _P]),
    "cfdb_batch_run": (_I, [_P, _P, _P, _I32, _I]),
    "cfdb_batch_launch_count": (_I, [_P, _PI64]),
    "cfdb_wave_adjoint_step": (_I, [_P, _P, _I, _I, _P, _P, _P, _P, _P, _D]),
    "cfdb_wave_gradient": (_I, [_P, _P, _I, _I, _P, _P, _P, _I32, _D, _I32, _PD, _P, _P, C.POINTER(GradientStats)]),
    "cfdb_wave_objective": (_I, [_P, _P, _I, _I, _P, _P, _P, _I32, _D, _PD]),
    "cfdb_revolve_plan": (_I, [_I32, _I32, _P, _P, _P, _I64, _PI64, _PI64]),
}


def header_functions(path: str = HEADER_PATH) -> list[str]:
    """Names of every function include/cfdb.h declares."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cfdb_[a-z0-9_]+)\s*\(", text)))


class CfdbError(RuntimeError):
    def __init__(self, code: int, msg: str, fn: str = ""):
        super().__init__(f"{fn}: status {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """Loads the in-tree libcfdb.so (fails loudly when it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libcfdb.so is not built ({LIB_PATH}); run `python -m cfdarcov2_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error(ctx=None) -> str:
    s = lib().cfdb_last_error(ctx)
    return s.decode() if s else ""


def check(rc: int, ctx=None, fn: str = "") -> None:
    if rc != OK:
        raise CfdbError(rc, last_error(ctx), fn)


def call(name: str, *args, ctx=None):
    rc = getattr(lib(), name)(*args)
    check(rc, ctx, name)
