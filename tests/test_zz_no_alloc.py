"""The allocation-free total (cfdb_total_fp64_noalloc), called through the C
ABI, against the regular entry point (cfdb_total_fp64).

It exists for callers that may not allocate device memory themselves, for
example a plugin whose host application owns every device allocation, or a
step recorded into another framework's CUDA graph.  Its reduction scratch is
a fixed array inside the library.  This file is named so that pytest collects
it last.  It passes when run alone in a fresh process and after the rest of
the suite."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

MAX_CELLS = 65536 * 4096


def noalloc_total(cfdb, field, volume, n=None):
    out = torch.full((1,), float("nan"), dtype=torch.float64, device=field.device)
    dtype = cfdb.F64 if field.dtype == torch.float64 else cfdb.F32
    stream = torch.cuda.current_stream(field.device).cuda_stream
    rc = cfdb.lib().cfdb_total_fp64_noalloc(dtype, C.c_void_p(field.data_ptr()), None, float(volume),
                                            int(field.numel() if n is None else n), C.c_void_p(stream),
                                            C.c_void_p(out.data_ptr()))
    return rc, out


def test_noalloc_total_matches_regular_entry_on_two_calls(cfdb):
    ctx = cfdb.Context(0)
    rng = np.random.default_rng(21)
    cases = [((40, 33, 20), np.float64), ((64, 50, 36), np.float32)]  # two calls in a row, different sizes/dtypes
    for (nx, ny, nz), ndt in cases:
        dx, dy, dz = 1 / nx, 1 / ny, 1 / nz
        mesh = cfdb.Mesh.structured(ctx, nx, ny, nz, dx, dy, dz)
        f = torch.tensor(rng.uniform(-1, 2, nx * ny * nz).astype(ndt), device="cuda:0")
        rc, out = noalloc_total(cfdb, f, dx * dy * dz)
        assert rc == 0, cfdb.capi.last_error()
        torch.cuda.synchronize()
        ref = ctx.total_fp64(mesh, f)
        assert float(out.item()) == pytest.approx(ref, rel=1e-14)
    ctx.close()


def test_noalloc_total_rejects_sizes_beyond_its_scratch(cfdb):
    f = torch.zeros(16, dtype=torch.float32, device="cuda:0")
    rc, out = noalloc_total(cfdb, f, 1.0, n=MAX_CELLS + 1)
    assert rc == cfdb.capi.EINVAL
    assert "maximum" in cfdb.capi.last_error()
    torch.cuda.synchronize()
    assert torch.isnan(out).all()  # nothing was launched
