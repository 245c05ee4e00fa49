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


def noalloc_total(cfdb, field, volume, n=None, volumes=None, field_ptr=None, out=None):
    if out is None:
        out = torch.full((1,), float("nan"), dtype=torch.float64, device=field.device)
    dtype = cfdb.F64 if field.dtype == torch.float64 else cfdb.F32
    stream = torch.cuda.current_stream(field.device).cuda_stream
    fp = C.c_void_p(field.data_ptr()) if field_ptr is None else field_ptr
    vp = None if volumes is None else C.c_void_p(volumes.data_ptr())
    rc = cfdb.lib().cfdb_total_fp64_noalloc(dtype, fp, vp, float(volume),
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


def test_noalloc_total_per_cell_volumes_on_a_distorted_mesh(cfdb):
    """The per-cell volume branch: the mesh's own volumes passed in, against
    the regular entry point on the same vertex mesh, twice in a row."""
    from cfdarcov2_b200.workloads import jittered_vertices
    ctx = cfdb.Context(0)
    n = 24
    mesh = cfdb.Mesh.from_vertices(ctx, n, n, n, 1 / n, 1 / n, 1 / n, jittered_vertices(n, seed=8))
    vol = torch.tensor(mesh.geometry(cfdb.capi.GEOM_VOLUME), dtype=torch.float64, device="cuda:0")
    rng = np.random.default_rng(5)
    for _ in range(2):
        f = torch.tensor(rng.uniform(-1, 2, mesh.n), dtype=torch.float64, device="cuda:0")
        rc, out = noalloc_total(cfdb, f, float("nan"), volumes=vol)
        assert rc == 0, cfdb.capi.last_error()
        torch.cuda.synchronize()
        assert float(out.item()) == pytest.approx(ctx.total_fp64(mesh, f), rel=1e-14)
    ctx.close()


def test_noalloc_total_of_no_cells_is_zero(cfdb):
    f = torch.ones(8, dtype=torch.float32, device="cuda:0")
    rc, out = noalloc_total(cfdb, f, 1.0)  # fills the scratch with a non-zero total first
    assert rc == 0
    rc, out = noalloc_total(cfdb, f, 1.0, n=0)
    assert rc == 0, cfdb.capi.last_error()
    torch.cuda.synchronize()
    assert float(out.item()) == 0.0


def test_noalloc_total_rejects_null_field_and_non_finite_volume(cfdb):
    f = torch.ones(8, dtype=torch.float32, device="cuda:0")
    rc, _ = noalloc_total(cfdb, f, 1.0, field_ptr=C.c_void_p(0))
    assert rc == cfdb.capi.EINVAL and "field is NULL" in cfdb.capi.last_error()
    rc, _ = noalloc_total(cfdb, f, float("inf"))
    assert rc == cfdb.capi.EINVAL and "finite" in cfdb.capi.last_error()


def test_noalloc_total_leaves_free_device_memory_unchanged(cfdb):
    """After a first call (which resolves the scratch address), further calls
    take no device memory: the driver's free-memory count does not move."""
    f = torch.rand(1 << 22, dtype=torch.float32, device="cuda:0")
    out = torch.empty(1, dtype=torch.float64, device="cuda:0")  # every buffer exists before the count
    rc, _ = noalloc_total(cfdb, f, 0.5, out=out)
    assert rc == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        rc, _ = noalloc_total(cfdb, f, 0.5, out=out)
        assert rc == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert float(out.item()) == pytest.approx(0.5 * float(f.double().sum()), rel=1e-12)


def test_noalloc_total_records_into_a_cuda_graph(cfdb):
    """After a first call, a call recorded into a CUDA graph (where any device
    allocation would end the capture with an error) replays with the field's
    current values."""
    ctx = cfdb.Context(0)
    nx, ny, nz = 48, 40, 36
    dx, dy, dz = 1 / nx, 1 / ny, 1 / nz
    mesh = cfdb.Mesh.structured(ctx, nx, ny, nz, dx, dy, dz)
    f = torch.rand(nx * ny * nz, dtype=torch.float32, device="cuda:0")
    out = torch.empty(1, dtype=torch.float64, device="cuda:0")
    rc, _ = noalloc_total(cfdb, f, dx * dy * dz, out=out)  # resolves the scratch address
    assert rc == 0, cfdb.capi.last_error()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        rc, _ = noalloc_total(cfdb, f, dx * dy * dz, out=out)
    assert rc == 0, cfdb.capi.last_error()
    for seed in (3, 4):
        gen = torch.Generator(device="cuda:0").manual_seed(seed)
        f.copy_(torch.rand(f.numel(), dtype=torch.float32, device="cuda:0", generator=gen) - 0.25)
        out.fill_(float("nan"))
        g.replay()
        torch.cuda.synchronize()
        assert float(out.item()) == pytest.approx(ctx.total_fp64(mesh, f), rel=1e-14)
    del g
    ctx.close()
