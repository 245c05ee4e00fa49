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
