"""Run-time compiled kernels through the C ABI (cfdb_kernel_build[_many] /
cfdb_kernel_launch, the role of the reference's KernelBuilder,
src/fvm3d.cpp:1219-1394): a batch compiles and runs, the operator templates
of cfdb_jit.cuh over the face arrays match cfdb_op_lapl / cfdb_op_grad bit for
bit, errors come back as status codes with the compiler log, and the on-disk
cache serves a later context and survives a damaged entry."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest
import torch

from cfdarcov2_b200 import capi

pytestmark = pytest.mark.gpu

DEV = "cuda:0"

AXPY = r"""
extern "C" __global__ void axpy(float a, const float* x, float* y, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = a * x[i] + y[i];
}
"""
SCALE = r"""
extern "C" __global__ void scale(float a, float* y, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = a * y[i];
}
"""
# the header's operator templates over the mesh's face arrays
OPERATORS = r"""
#include "cfdb_jit.cuh"
extern "C" __global__ void ops(CfdbGeom g, const float* phi, float* lap, float* grd) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.n) return;
  auto f = [&](long long j) { return phi[j]; };
  lap[i] = cfdb_lapl(f, i, 7, g);
  grd[i] = cfdb_grad(f, i, 3, g);
}
"""


def build_many(ctx, sources, names):
    n = len(sources)
    src = (C.c_char_p * n)(*[s.encode() for s in sources])
    nm = (C.c_char_p * n)(*[s.encode() for s in names])
    out = (C.c_void_p * n)()
    capi.call("cfdb_kernel_build_many", ctx.h, n, src, nm, out, ctx=ctx.h)
    return [C.c_void_p(out[k]) for k in range(n)]


def launch(ctx, k, n, *args):
    arr = (C.c_void_p * len(args))(*[C.cast(C.pointer(a), C.c_void_p) for a in args])
    capi.call("cfdb_kernel_launch", k, int(n), 128, arr, ctx=ctx.h)


def test_batch_build_and_launch(cfdb):
    ctx = cfdb.Context(0)
    k_axpy, k_scale = build_many(ctx, [AXPY, SCALE], ["axpy", "scale"])
    n = 1000
    x = torch.arange(n, dtype=torch.float32, device=DEV)
    y = torch.ones(n, dtype=torch.float32, device=DEV)
    launch(ctx, k_axpy, n, C.c_float(2.0), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), C.c_longlong(n))
    launch(ctx, k_scale, n, C.c_float(0.5), C.c_void_p(y.data_ptr()), C.c_longlong(n))
    ctx.sync()
    assert torch.equal(y.cpu(), (2 * torch.arange(n, dtype=torch.float32) + 1) * 0.5)
    for k in (k_axpy, k_scale):
        capi.call("cfdb_kernel_destroy", k)


def test_header_operators_equal_the_operator_kernels(cfdb):
    ctx = cfdb.Context(0)
    m = cfdb.Mesh.structured(ctx, 12, 10, 9, 1 / 12, 0.1, 1 / 9)
    g = capi.PlainGeometry()
    capi.call("cfdb_mesh_plain_geometry", m.h, C.byref(g), ctx=ctx.h)
    (k,) = build_many(ctx, [OPERATORS], ["ops"])
    rng = np.random.default_rng(3)
    phi = torch.tensor(rng.standard_normal(m.n), dtype=torch.float32, device=DEV)
    lap, grd = torch.empty_like(phi), torch.empty_like(phi)
    launch(ctx, k, m.n, g, C.c_void_p(phi.data_ptr()), C.c_void_p(lap.data_ptr()), C.c_void_p(grd.data_ptr()))
    ctx.sync()
    assert torch.equal(lap, ctx.lapl(m, phi, mask=7))
    assert torch.equal(grd, ctx.grad(m, phi, mask=3))


def test_compile_errors_and_missing_entry(cfdb):
    ctx = cfdb.Context(0)
    with pytest.raises(capi.CfdbError) as e:
        build_many(ctx, ["extern \"C\" __global__ void bad( { }"], ["bad"])
    assert e.value.code == capi.EINVAL and "does not compile" in str(e.value)
    with pytest.raises(capi.CfdbError) as e:
        build_many(ctx, [AXPY], ["no_such_kernel"])
    assert e.value.code == capi.EINVAL
    # the context stays usable
    (k,) = build_many(ctx, [SCALE], ["scale"])
    y = torch.full((64,), 3.0, device=DEV)
    launch(ctx, k, 64, C.c_float(2.0), C.c_void_p(y.data_ptr()), C.c_longlong(64))
    ctx.sync()
    assert torch.all(y == 6.0)


def test_disk_cache_serves_a_new_context_and_survives_damage(cfdb, tmp_path, monkeypatch):
    monkeypatch.setenv("CFDB_KERNEL_CACHE", str(tmp_path))
    src = AXPY.replace("axpy", "axpy_cached")
    ctx1 = cfdb.Context(0)
    build_many(ctx1, [src], ["axpy_cached"])
    entries = list(tmp_path.glob("*.cubin"))
    assert len(entries) == 1 and entries[0].stat().st_size > 100
    # a new context (no in-memory module) loads it; a truncated entry is recompiled and rewritten
    ctx2 = cfdb.Context(0)
    build_many(ctx2, [src], ["axpy_cached"])
    with open(entries[0], "r+b") as f:
        f.truncate(40)
    ctx3 = cfdb.Context(0)
    (k,) = build_many(ctx3, [src], ["axpy_cached"])
    assert entries[0].stat().st_size > 100
    n = 256
    x = torch.ones(n, device=DEV)
    y = torch.zeros(n, device=DEV)
    launch(ctx3, k, n, C.c_float(4.0), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), C.c_longlong(n))
    ctx3.sync()
    assert torch.all(y == 4.0)
    monkeypatch.setenv("CFDB_KERNEL_CACHE", "off")
    ctx4 = cfdb.Context(0)
    build_many(ctx4, [src.replace("axpy_cached", "axpy_uncached")], ["axpy_uncached"])
    assert len(list(tmp_path.glob("*.cubin"))) == 1
    assert os.environ["CFDB_KERNEL_CACHE"] == "off"


def test_kernel_info_reports_the_built_kernel(cfdb):
    ctx = cfdb.Context(0)
    (k,) = build_many(ctx, [AXPY.replace("axpy", "axpy_info")], ["axpy_info"])
    regs, local, maxt = C.c_int(0), C.c_int64(-1), C.c_int(0)
    capi.call("cfdb_kernel_info", k, C.byref(regs), C.byref(local), C.byref(maxt), ctx=ctx.h)
    assert 0 < regs.value <= 255 and local.value == 0 and maxt.value >= 128
    capi.call("cfdb_kernel_destroy", k)
    with pytest.raises(capi.CfdbError) as e:
        capi.call("cfdb_kernel_info", None, None, None, None)
    assert e.value.code == capi.EINVAL
