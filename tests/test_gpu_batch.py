"""Batched ensemble of independent cubes (heat or wave, uneven sizes and
parameters) in one persistent launch per step: every problem matches the
FP64 oracle run on its own mesh; graph replay equals eager launches; the
autotuner picks a configuration and caches it."""
from __future__ import annotations

import json

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def problems():
    from cfdarcov2_b200.workloads import ensemble_problems
    return ensemble_problems(count=10, nmin=5, nmax=18, seed=11)


@pytest.mark.parametrize("cfg", [(256, 128, 4), (32, 32, 2), (8192, 64, 8)])
def test_ensemble_matches_oracle_per_problem(cfdb, oracle, ctx, cfg):
    """Work items of one plane, a few planes, and whole problems (more
    planes than n); column runs shorter and longer than n^2."""
    from cfdarcov2_b200.workloads import ensemble_initial
    probs = problems()
    b = cfdb.Batch(ctx, probs)
    pool0 = ensemble_initial(probs, b.offsets, b.pool_elems)
    rng = np.random.default_rng(5)
    for p, off in zip(probs, b.offsets):  # give the wave velocities something to do
        if p["kind"] == 1:
            n3 = p["n"] ** 3
            pool0[off + n3: off + 4 * n3] = rng.standard_normal(3 * n3) * 0.1
    a = torch.tensor(pool0, device=DEV)
    c = torch.empty_like(a)
    steps = 13
    b.set_config(*cfg)
    b.run(a, c, steps, use_graph=True)
    got = (c if steps % 2 else a).cpu().numpy()
    assert b.launch_count() == steps
    for p, off in zip(probs, b.offsets):
        n = p["n"]
        m = oracle.Mesh(n, n, n, 1 / n, 1 / n, 1 / n)
        if p["kind"] == 0:
            ref = m.heat_solve(pool0[off: off + n ** 3].astype(np.float64), p["param"], p["dt"], steps)
            g = got[off: off + n ** 3]
        else:
            ref = m.wave_solve(pool0[off: off + 4 * n ** 3].astype(np.float64), p["dt"], steps, cconst=p["param"])
            g = got[off: off + 4 * n ** 3]
        assert rel_l2(g, ref) <= 1e-5, (p["n"], p["kind"])


def test_graph_replay_equals_eager(cfdb, ctx):
    from cfdarcov2_b200.workloads import ensemble_initial
    probs = problems()
    b = cfdb.Batch(ctx, probs)
    pool0 = torch.tensor(ensemble_initial(probs, b.offsets, b.pool_elems), device=DEV)
    for cfg in [(128, 64, 2), (1024, 256, 8), (4096, 512, 4)]:
        b.set_config(*cfg)
        a1, c1 = pool0.clone(), torch.empty_like(pool0)
        b.run(a1, c1, 8, use_graph=False)
        a2, c2 = pool0.clone(), torch.empty_like(pool0)
        b.run(a2, c2, 8, use_graph=True)
        torch.cuda.synchronize()
        assert torch.equal(a1, a2), cfg


def test_autotuner_caches_choice(cfdb, ctx, tmp_path):
    from cfdarcov2_b200.workloads import ensemble_initial
    probs = problems()
    b = cfdb.Batch(ctx, probs)
    pool0 = torch.tensor(ensemble_initial(probs, b.offsets, b.pool_elems), device=DEV)
    a, c = pool0.clone(), torch.empty_like(pool0)
    cache = tmp_path / "tune.json"
    b.tune(a, c, cache)
    chosen = b.get_config()
    data = json.loads(cache.read_text())
    assert len(data) == 1 and list(data.values())[0][:3] == list(chosen)
    assert list(data.values())[0][3] in (0, 1, 2)  # the kernel form that won
    b2 = cfdb.Batch(ctx, probs)
    b2.tune(a, c, cache)  # served from the cache
    assert b2.get_config() == chosen


def test_batch_rejects_bad_problems(cfdb, ctx):
    with pytest.raises(cfdb.CfdbError):
        cfdb.Batch(ctx, [dict(n=1, kind=0, param=0.01, dt=1e-3)])
    with pytest.raises(cfdb.CfdbError):
        cfdb.Batch(ctx, [dict(n=8, kind=2, param=0.01, dt=1e-3)])
    b = cfdb.Batch(ctx, [dict(n=8, kind=0, param=0.01, dt=1e-3)])
    with pytest.raises(cfdb.CfdbError):
        b.set_config(256, 100, 4)


def cells(pool, b, probs):
    """The problems' cells of a pool, without the spare floats around them
    (scratch the kernels may read but never write)."""
    return torch.cat([pool[off: off + p["n"] ** 3 * (1 if p["kind"] == 0 else 4)] for p, off in zip(probs, b.offsets)])


def mixed_problems():
    from cfdarcov2_b200.workloads import ensemble_problems
    return ensemble_problems(count=40, nmin=5, nmax=70, seed=17)


@pytest.mark.parametrize("cfg", [(2048, 128, 4), (8192, 256, 2), (32768, 512, 1), (256, 256, 3)])
def test_staged_ring_equals_column_march_bitwise(cfdb, ctx, cfg):
    """The staged kernel (a producer warp streaming plane rows into a
    shared-memory ring, consumer warps marching the columns) gives the column
    march's bits: items shorter and longer than n, column runs shorter and
    longer than n^2, 1-4 CTAs per SM; the wave velocities are non-zero."""
    from cfdarcov2_b200.workloads import ensemble_initial
    probs = mixed_problems()
    b = cfdb.Batch(ctx, probs)
    pool0 = ensemble_initial(probs, b.offsets, b.pool_elems)
    rng = np.random.default_rng(9)
    for p, off in zip(probs, b.offsets):
        if p["kind"] == 1:
            n3 = p["n"] ** 3
            pool0[off + n3: off + 4 * n3] = rng.standard_normal(3 * n3) * 0.1
    b.set_config(*cfg)
    outs = []
    for form, graph in ((1, True), (1, False), (0, False), (2, True)):
        b.set_staged(form)
        a = torch.tensor(pool0, device=DEV)
        c = torch.full_like(a, float("nan"))  # NaN in the spare floats must never reach a cell
        outs.append(cells(b.run(a, c, 9, use_graph=graph), b, probs).clone())
    ctx.sync()
    assert not torch.isnan(outs[2]).any()
    assert all(torch.equal(o, outs[2]) for o in outs)
    with pytest.raises(cfdb.CfdbError):
        b.set_staged(3)
