"""The benchmark workloads at their own sizes: the FP32 fused path against the
FP64 plain GPU path, which is bit-identical to the FP64 oracle on every case
the oracle can run in seconds (tests/test_gpu_ops.py, test_gpu_euler.py).

  * ensemble: 512 cubes, n log-uniform in [16, 96] (seed 4), 300 steps, every
    problem checked on its own (rel L2 <= 1e-5);
  * distorted wave: 128^3 on vertices jittered by U(-0.2, 0.2) dx (seed 2),
    500 steps (rel L2 <= 1e-5);
  * Sod: 512 x 64 x 64 to t = 0.2 (rel L2 <= 1e-5), FP64 totals of mass and
    energy conserved (the waves stay inside the tube until t = 0.2).

Each pins the d1t update (src/fvm3d.cpp:675-708) of its workload at the size
that is measured."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TOL = 1e-5  # rel L2, FP32 fused vs FP64


def test_ensemble_config_every_problem_vs_fp64_plain(cfdb, ctx):
    from cfdarcov2_b200.workloads import ensemble_initial, ensemble_problems
    probs = ensemble_problems()  # 512 problems, n in [16, 96], seed 4
    assert len(probs) == 512
    steps = 300
    b = cfdb.Batch(ctx, probs)
    pool0 = ensemble_initial(probs, b.offsets, b.pool_elems)
    a = torch.tensor(pool0, device=DEV)
    c = torch.empty_like(a)
    b.run(a, c, steps, use_graph=True)  # the library's default (or cached tuned) configuration
    got = (c if steps % 2 else a).cpu().numpy()
    worst = 0.0
    for p, off in zip(probs, b.offsets):
        n = p["n"]
        n3 = n ** 3
        m = cfdb.Mesh.structured(ctx, n, n, n, 1 / n, 1 / n, 1 / n)
        if p["kind"] == 0:
            x = torch.tensor(pool0[off: off + n3], dtype=torch.float64, device=DEV)
            ref = ctx.heat_run(m, x, torch.empty_like(x), p["param"], p["dt"], steps, path=cfdb.PLAIN)
            g = got[off: off + n3]
        else:
            x = torch.tensor(pool0[off: off + 4 * n3], dtype=torch.float64, device=DEV)
            ref = ctx.wave_run(m, x, torch.empty_like(x), p["dt"], steps, c_const=p["param"], path=cfdb.PLAIN)
            g = got[off: off + 4 * n3]
        err = rel_l2(g, ref.cpu().numpy())
        worst = max(worst, err)
        assert err <= TOL, (n, p["kind"], err)
        m.close()
    print(f"ensemble worst rel L2 {worst:.3e}")


def test_distorted_wave_config_vs_fp64_plain(cfdb, ctx):
    from cfdarcov2_b200.workloads import jittered_vertices, wave_config
    cfg = wave_config(n=128, steps=500)
    n, T = cfg["n"], cfg["steps"]
    m = cfdb.Mesh.from_vertices(ctx, n, n, n, cfg["dx"], cfg["dx"], cfg["dx"], jittered_vertices(n, seed=2))
    dt = m.wave_dt(0.4)
    outs = {}
    for name, tdt, path in (("f32", torch.float32, cfdb.FUSED), ("f64", torch.float64, cfdb.PLAIN)):
        q = torch.tensor(cfg["q0"], dtype=tdt, device=DEV)
        outs[name] = ctx.wave_run(m, q, torch.empty_like(q), dt, T, path=path).double().cpu().numpy()
    err = rel_l2(outs["f32"], outs["f64"])
    print(f"distorted wave 128^3 x 500: rel L2 {err:.3e}")
    assert err <= TOL
    # the pulse has spread: the solve is not a near-identity
    assert rel_l2(outs["f64"], cfg["q0"]) > 0.1


def test_sod_config_vs_fp64_plain_and_totals(cfdb, ctx):
    from cfdarcov2_b200.workloads import sod_config
    cfg = sod_config()
    nx, ny, nz = cfg["nx"], cfg["ny"], cfg["nz"]
    m = cfdb.Mesh.structured(ctx, nx, ny, nz, cfg["dx"], cfg["dy"], cfg["dz"])
    res = {}
    for name, dty, tdt, path in (("f32", cfdb.F32, torch.float32, cfdb.FUSED),
                                 ("f64", cfdb.F64, torch.float64, cfdb.PLAIN)):
        e = cfdb.Euler(ctx, m, dtype=dty, path=path, gamma=cfg["gamma"], cfl=cfg["cfl"], t_end=cfg["t_end"],
                       max_steps=20000)
        a = torch.tensor(cfg["U0"], dtype=tdt, device=DEV)
        b = torch.empty_like(a)
        e.begin(a)
        steps, in_b = e.run(a, b, 64)
        t, _, fin = e.status()
        assert fin and t == cfg["t_end"]
        res[name] = ((b if in_b else a).double().cpu().numpy(), steps, e.totals())
        e.close()
    assert abs(res["f32"][1] - res["f64"][1]) <= 1
    err = rel_l2(res["f32"][0], res["f64"][0])
    print(f"Sod 512x64x64: {res['f32'][1]} steps, rel L2 {err:.3e}")
    assert err <= TOL
    for name, bound in (("f32", 2e-6), ("f64", 1e-12)):
        tot = res[name][2]
        assert tot.shape[0] == res[name][1] + 1
        for col in (0, 1):  # mass, energy
            drift = np.abs(tot[:, col] - tot[0, col]).max() / tot[0, col]
            assert drift <= bound, (name, col, drift)
