"""The bounded device wait of the TMA sweep runs out and reports, without any
fault: a test hook arms one plane's barrier in the first CTA (its first
interior plane, which every x chunk has) with the plane's byte count but
issues no copy for it (a completion that never
comes), with the wait bound lowered to 1e6 SM cycles (about 0.5 ms).  The
launch must end by itself, cfdb_sync must return CFDB_ETIMEOUT, and the same
context must then run a normal step with the correct result.  (The
reference has no device waits; any CUDA error exits its process through
gpuAssert, include/cuda_operators.hpp:29-36.)"""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.mark.parametrize("kind", ["wave", "heat"])
def test_wait_runs_out_and_context_recovers(cfdb, kind):
    ctx = cfdb.Context(0)
    n = 32
    m = cfdb.Mesh.structured(ctx, n, n, n, 1 / n, 1 / n, 1 / n)
    rng = np.random.default_rng(12)
    nf = 4 if kind == "wave" else 1
    q = torch.tensor(rng.standard_normal(nf * m.n), dtype=torch.float32, device=DEV)

    def step(out):
        if kind == "wave":
            ctx.wave_step(m, q, out, 0.4 / (3 * n), path=cfdb.FUSED)
        else:
            ctx.heat_step(m, q, out, 0.01, 0.1 / (n * n) / 0.01, path=cfdb.FUSED)

    good = torch.empty_like(q)
    step(good)
    ctx.sync()

    ctx.set_wait_limit(1_000_000, missing_plane=1)  # plane 1 (x = x0) exists in every CTA's chunk
    bad = torch.zeros_like(q)
    step(bad)
    with pytest.raises(cfdb.CfdbError) as ei:
        ctx.sync()
    assert ei.value.code == cfdb.capi.ETIMEOUT
    assert "bounded device wait" in str(ei.value)

    ctx.set_wait_limit()  # default bound, hook off
    again = torch.empty_like(q)
    step(again)
    ctx.sync()  # the error word was cleared when it was reported
    assert torch.equal(again, good)
    ctx.close()


def test_wait_limit_rejects_bad_arguments(cfdb, ctx):
    with pytest.raises(cfdb.CfdbError):
        ctx.set_wait_limit(10)
    with pytest.raises(cfdb.CfdbError):
        ctx.set_wait_limit(1_000_000, missing_plane=-2)


@pytest.mark.parametrize("kind", ["distorted", "euler"])
def test_face_sweep_wait_runs_out_and_context_recovers(cfdb, kind):
    """The same on the face-flux sweep (its own staging: the ghost plane's
    geometry copy of a vertex mesh, derived values for Euler): the launch
    ends by itself, cfdb_sync reports CFDB_ETIMEOUT, and the context then
    runs the step with the correct result."""
    ctx = cfdb.Context(0)
    if kind == "distorted":
        from cfdarcov2_b200.workloads import jittered_vertices
        n = 32
        m = cfdb.Mesh.from_vertices(ctx, n, n, n, 1 / n, 1 / n, 1 / n, jittered_vertices(n, seed=2))
        q = torch.tensor(np.random.default_rng(13).standard_normal(4 * m.n), dtype=torch.float32, device=DEV)

        def run(out):
            ctx.wave_step(m, q, out, 0.4 / (3 * n), path=cfdb.FUSED)
            return out
    else:
        from cfdarcov2_b200.workloads import sod_state
        U0, (dx, dy, dz) = sod_state(64, 8, 8, 1.0, 0.125)
        m = cfdb.Mesh.structured(ctx, 64, 8, 8, dx, dy, dz)
        e = cfdb.Euler(ctx, m, dtype=cfdb.F32, path=cfdb.FUSED, gamma=1.4, cfl=0.4, t_end=0.2, max_steps=1000)
        q = torch.tensor(U0, dtype=torch.float32, device=DEV)

        def run(out):
            a = q.clone()
            e.begin(a)
            for k in range(4):
                e.step(a, out) if k % 2 == 0 else e.step(out, a)
            return a

    good = run(torch.empty_like(q)).clone()
    ctx.sync()

    ctx.set_wait_limit(1_000_000, missing_plane=1)
    run(torch.zeros_like(q))
    with pytest.raises(cfdb.CfdbError) as ei:
        ctx.sync()
    assert ei.value.code == cfdb.capi.ETIMEOUT

    ctx.set_wait_limit()
    again = run(torch.empty_like(q)).clone()
    ctx.sync()
    assert torch.equal(again, good)
    if kind == "euler":
        e.close()
    ctx.close()


def test_resident_heat_wait_runs_out_and_context_recovers(cfdb):
    """The cluster-resident heat solver on several clusters: with the hook
    one cluster never publishes step 3's edge planes, so its neighbours'
    bounded waits run out; the launch ends by itself (later waits are
    skipped), cfdb_sync reports CFDB_ETIMEOUT, and the context then runs the
    solve with the per-step sweep's result."""
    ctx = cfdb.Context(0)
    X, n = 128, 64  # too large for one cluster: four clusters of 16 CTAs, two planes each
    m = cfdb.Mesh.structured(ctx, X, n, n, 1 / X, 1 / n, 1 / n)
    T0 = torch.tensor(np.random.default_rng(14).uniform(0, 1, m.n), dtype=torch.float32, device=DEV)
    k, dt, steps = 0.01, 0.1 / (X * X) / 0.01, 8
    ref_a, ref_b = T0.clone(), torch.empty_like(T0)
    p, q = ref_a, ref_b
    for _ in range(steps):
        ctx.heat_step(m, p, q, k, dt)
        p, q = q, p
    ctx.sync()

    ctx.set_wait_limit(1_000_000, missing_plane=3)
    a, b = T0.clone(), torch.empty_like(T0)
    ctx.heat_run(m, a, b, k, dt, steps)
    with pytest.raises(cfdb.CfdbError) as ei:
        ctx.sync()
    assert ei.value.code == cfdb.capi.ETIMEOUT

    ctx.set_wait_limit()
    a, b = T0.clone(), torch.empty_like(T0)
    final = ctx.heat_run(m, a, b, k, dt, steps)
    ctx.sync()
    assert torch.equal(final, p)
    ctx.close()
