"""Run-to-run determinism of the fused paths (the reference has no race
detection; compute-sanitizer is not available here, so a kernel that races
on its inputs or reduces in a timing-dependent order would show up as two
runs of the same inputs that differ), and the Euler run's health check:
a NaN in the state stops the run with CFDB_ENUMERIC instead of letting a
non-finite dt end it early."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def test_fused_wave_and_heat_runs_repeat_bit_for_bit(cfdb, ctx):
    from cfdarcov2_b200.workloads import wave_config
    n = 64
    cfg = wave_config(n=n, steps=40)
    m = cfdb.Mesh.structured(ctx, n, n, n, cfg["dx"], cfg["dx"], cfg["dx"])
    q0 = torch.tensor(cfg["q0"], dtype=torch.float32, device=DEV)
    outs = []
    for _ in range(2):
        a, b = q0.clone(), torch.empty_like(q0)
        outs.append(ctx.wave_run(m, a, b, cfg["dt"], 40, c_const=cfg["c"], path=cfdb.FUSED).clone())
    assert torch.equal(outs[0], outs[1])
    T0 = torch.rand(m.n, device=DEV)
    res = []
    for _ in range(2):
        a, b = T0.clone(), torch.empty_like(T0)
        res.append(ctx.heat_run(m, a, b, 0.01, 1e-5, 30, path=cfdb.FUSED).clone())
    assert torch.equal(res[0], res[1])


def test_euler_fused_run_and_totals_repeat_bit_for_bit(cfdb, ctx):
    """The device-side dt (max reduction) and the FP64 totals (fixed-order
    merge of per-CTA partials) give the same bits every run."""
    from cfdarcov2_b200.workloads import sod_state
    nx, ny, nz = 256, 16, 16
    U0, (dx, dy, dz) = sod_state(nx, ny, nz)
    m = cfdb.Mesh.structured(ctx, nx, ny, nz, dx, dy, dz)
    runs = []
    for _ in range(2):
        e = cfdb.Euler(ctx, m, dtype=cfdb.F32, path=cfdb.FUSED, gamma=1.4, cfl=0.4, t_end=0.05, max_steps=10000)
        a = torch.tensor(U0, dtype=torch.float32, device=DEV)
        b = torch.empty_like(a)
        e.begin(a)
        steps, in_b = e.run(a, b, 32)
        runs.append((steps, (b if in_b else a).cpu(), e.totals()))
    assert runs[0][0] == runs[1][0]
    assert torch.equal(runs[0][1], runs[1][1])
    assert np.array_equal(runs[0][2], runs[1][2])


def test_ensemble_and_gradient_repeat_bit_for_bit(cfdb, ctx):
    from cfdarcov2_b200.workloads import adjoint_config, ensemble_initial, ensemble_problems
    probs = ensemble_problems(count=12, nmin=8, nmax=24, seed=3)
    bt = cfdb.Batch(ctx, probs)
    pool0 = torch.tensor(ensemble_initial(probs, bt.offsets, bt.pool_elems), device=DEV)
    res = []
    for _ in range(2):
        a, c = pool0.clone(), torch.empty_like(pool0)
        bt.run(a, c, 20, use_graph=True)
        res.append(a.clone())  # an even step count ends in the first buffer
    assert torch.equal(res[0], res[1])

    cfg = adjoint_config(n=32, steps=24)
    n, T, dt = cfg["n"], cfg["steps"], cfg["dt"]
    m = cfdb.Mesh.structured(ctx, n, n, n, 1 / n, 1 / n, 1 / n)
    q0 = torch.tensor(cfg["q0"], dtype=torch.float32, device=DEV)
    cc = torch.tensor(cfg["c"], dtype=torch.float32, device=DEV)
    tgt = torch.tensor(cfg["q0"][: m.n], dtype=torch.float32, device=DEV) * 0.5
    grads = []
    for _ in range(2):
        g_c, g_p = torch.empty(m.n, device=DEV), torch.empty(m.n, device=DEV)
        J, _ = ctx.wave_gradient(m, q0, cc, tgt, T, dt, T, g_c, g_p, path=cfdb.FUSED)
        grads.append((J, g_c.cpu(), g_p.cpu()))
    assert grads[0][0] == grads[1][0]
    assert torch.equal(grads[0][1], grads[1][1]) and torch.equal(grads[0][2], grads[1][2])


def test_nan_in_the_state_stops_the_euler_run(cfdb, ctx):
    from cfdarcov2_b200.workloads import sod_state
    nx, ny, nz = 128, 8, 8
    U0, (dx, dy, dz) = sod_state(nx, ny, nz)
    U0 = U0.copy()
    U0[nx * ny * nz // 2 + 5] = np.nan  # one density value, injected on the host
    m = cfdb.Mesh.structured(ctx, nx, ny, nz, dx, dy, dz)
    e = cfdb.Euler(ctx, m, dtype=cfdb.F32, path=cfdb.FUSED, gamma=1.4, cfl=0.4, t_end=0.2, max_steps=10000)
    a = torch.tensor(U0, dtype=torch.float32, device=DEV)
    b = torch.empty_like(a)
    e.begin(a)
    with pytest.raises(cfdb.capi.CfdbError) as err:
        e.run(a, b, 8)
    assert err.value.code == cfdb.capi.ENUMERIC and "not finite" in str(err.value)
    ctx.sync()  # the context stays usable
