"""Discrete adjoint of the wave step and the checkpointed gradient through
the C ABI, against the CPU oracle and finite differences."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def dev(a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


def setup(n, seed=3, verts=None):
    rng = np.random.default_rng(seed)
    c = np.exp(0.2 * rng.standard_normal(n ** 3))
    from cfdarcov2_b200.workloads import wave_state
    q0 = wave_state(n, sigma=0.15)
    target = rng.standard_normal(n ** 3) * 0.01
    return c, q0, target


@pytest.mark.parametrize("vert", [False, True])
def test_adjoint_step_plain_fp64_bitwise(cfdb, oracle, ctx, vert):
    from cfdarcov2_b200.workloads import jittered_vertices
    n = 7
    if vert:
        V = jittered_vertices(n, seed=4)
        m = cfdb.Mesh.from_vertices(ctx, n, n, n, 1 / n, 1 / n, 1 / n, V)
        o = oracle.Mesh(n, n, n, 1 / n, 1 / n, 1 / n, vertices=V)
    else:
        m = cfdb.Mesh.structured(ctx, n, n, n, 1 / n, 1 / n, 1 / n)
        o = oracle.Mesh(n, n, n, 1 / n, 1 / n, 1 / n)
    rng = np.random.default_rng(2)
    c = np.exp(0.2 * rng.standard_normal(m.n))
    q, lam1, gc0 = rng.standard_normal((3, 4 * m.n))
    gc0 = gc0[: m.n]
    dt = o.wave_dt(0.4, c=c)
    ref_lam0, ref_gc = o.wave_adjoint_step(q, lam1, c, gc0, dt)
    lam0 = torch.empty(4 * m.n, dtype=torch.float64, device=DEV)
    gc = dev(gc0, torch.float64)
    ctx.wave_adjoint_step(m, dev(q, torch.float64), dev(lam1, torch.float64), lam0, dev(c, torch.float64), gc, dt,
                          path=cfdb.PLAIN)
    assert np.array_equal(lam0.cpu().numpy(), ref_lam0)
    assert np.array_equal(gc.cpu().numpy(), ref_gc)


@pytest.mark.parametrize("shape", [(12, 12, 12), (20, 9, 16), (5, 17, 68), (7, 6, 10)])
def test_adjoint_step_fused_fp32_vs_oracle(cfdb, oracle, ctx, shape):
    """Sweep kernel (nz % 4 == 0; 32- and 64-wide z tiles, partial tiles,
    walls on every side) and the gather fallback (nz = 10)."""
    X, Y, Z = shape
    m = cfdb.Mesh.structured(ctx, X, Y, Z, 1 / X, 1 / Y, 1 / Z)
    o = oracle.Mesh(X, Y, Z, 1 / X, 1 / Y, 1 / Z)
    rng = np.random.default_rng(6)
    c = np.exp(0.2 * rng.standard_normal(m.n))
    q, lam1 = rng.standard_normal((2, 4 * m.n))
    gc0 = rng.standard_normal(m.n) * 1e-3
    dt = o.wave_dt(0.4, c=c)
    ref_lam0, ref_gc = o.wave_adjoint_step(q, lam1, c, gc0, dt)
    lam0 = torch.empty(4 * m.n, dtype=torch.float32, device=DEV)
    gc = dev(gc0, torch.float32)
    ctx.wave_adjoint_step(m, dev(q, torch.float32), dev(lam1, torch.float32), lam0, dev(c, torch.float32), gc, dt,
                          path=cfdb.FUSED)
    assert rel_l2(lam0.cpu().numpy(), ref_lam0) <= 1e-6
    assert rel_l2(gc.cpu().numpy(), ref_gc) <= 1e-5


def test_gpu_dot_product_fp64(cfdb, ctx):
    """<A v, w> = <v, A^T w> with the GPU forward and adjoint steps."""
    n = 10
    m = cfdb.Mesh.structured(ctx, n, n, n, 1 / n, 1 / n, 1 / n)
    rng = np.random.default_rng(8)
    c = dev(np.exp(0.2 * rng.standard_normal(m.n)), torch.float64)
    v = dev(rng.standard_normal(4 * m.n), torch.float64)
    w = dev(rng.standard_normal(4 * m.n), torch.float64)
    dt = m.wave_dt(0.4, c=c.cpu().numpy())
    Av = torch.empty_like(v)
    ctx.wave_step(m, v, Av, dt, c=c, speed_mode=1, path=cfdb.PLAIN)
    ATw = torch.empty_like(w)
    gc = torch.zeros(m.n, dtype=torch.float64, device=DEV)
    ctx.wave_adjoint_step(m, v, w, ATw, c, gc, dt, path=cfdb.PLAIN)
    assert float(torch.dot(Av, w)) == pytest.approx(float(torch.dot(v, ATw)), rel=1e-12)


def test_gradient_fp64_matches_oracle(cfdb, oracle, ctx):
    n, steps = 8, 12
    m = cfdb.Mesh.structured(ctx, n, n, n, 1 / n, 1 / n, 1 / n)
    o = oracle.Mesh(n, n, n, 1 / n, 1 / n, 1 / n)
    c, q0, target = setup(n)
    dt = o.wave_dt(0.4, c=c * 1.1)
    J, gc, gp = o.wave_gradient(q0, c, target, dt, steps)
    g_c = torch.empty(m.n, dtype=torch.float64, device=DEV)
    g_p = torch.empty(m.n, dtype=torch.float64, device=DEV)
    Jg, st = ctx.wave_gradient(m, dev(q0, torch.float64), dev(c, torch.float64), dev(target, torch.float64), steps,
                               dt, steps, g_c, g_p, path=cfdb.PLAIN)
    assert Jg == pytest.approx(J, rel=1e-13)
    assert np.array_equal(g_c.cpu().numpy(), gc) and np.array_equal(g_p.cpu().numpy(), gp)
    assert st.forward_steps == steps and st.adjoint_steps == steps


@pytest.mark.parametrize("snaps", [1, 2, 3, 5])
def test_revolve_gradient_equals_store_all(cfdb, ctx, snaps):
    """Recomputing from checkpoints reproduces the store-all gradient bit for
    bit (same kernels, same order) with only `snaps` state slots."""
    n, steps = 16, 23
    m = cfdb.Mesh.structured(ctx, n, n, n, 1 / n, 1 / n, 1 / n)
    c, q0, target = setup(n)
    dt = m.wave_dt(0.4, c=c * 1.1)
    args = [dev(q0, torch.float32), dev(c, torch.float32), dev(target, torch.float32)]
    outs = {}
    for s in (steps, snaps):
        g_c = torch.empty(m.n, device=DEV)
        g_p = torch.empty(m.n, device=DEV)
        J, st = ctx.wave_gradient(m, *args, steps, dt, s, g_c, g_p, path=cfdb.FUSED)
        outs[s] = (J, g_c.cpu(), g_p.cpu(), st.forward_steps)
    assert outs[snaps][0] == outs[steps][0]
    assert torch.equal(outs[snaps][1], outs[steps][1]) and torch.equal(outs[snaps][2], outs[steps][2])
    _, fwd = cfdb.revolve_plan(steps, snaps)
    assert outs[snaps][3] == fwd + 1 and outs[steps][3] == steps


def test_gradient_workspace_is_pooled(cfdb, ctx):
    """The checkpoint slots of a gradient come from the context's pool: after
    the call nothing stays counted as allocated, a second call reuses the
    cached blocks and gives the same result, and cfdb_ctx_trim releases them."""
    n, steps = 16, 9
    m = cfdb.Mesh.structured(ctx, n, n, n, 1 / n, 1 / n, 1 / n)
    c, q0, target = setup(n)
    dt = m.wave_dt(0.4, c=c * 1.1)
    args = [dev(q0, torch.float32), dev(c, torch.float32), dev(target, torch.float32)]
    before = ctx.allocated_bytes()
    res = []
    for _ in range(2):
        g_c, g_p = torch.empty(m.n, device=DEV), torch.empty(m.n, device=DEV)
        J, _ = ctx.wave_gradient(m, *args, steps, dt, steps, g_c, g_p, path=cfdb.FUSED)
        res.append((J, g_c.cpu(), g_p.cpu()))
        assert ctx.allocated_bytes() == before
    assert res[0][0] == res[1][0] and torch.equal(res[0][1], res[1][1]) and torch.equal(res[0][2], res[1][2])
    ctx.trim()
    J, _ = ctx.wave_gradient(m, *args, steps, dt, steps, g_c, g_p, path=cfdb.FUSED)
    assert J == res[0][0]


def test_gradient_fp32_vs_finite_differences_full_size(cfdb, ctx):
    """The adjoint workload at full size: 128^3, 400 steps, c = exp(0.2 g) with
    g a seeded Gaussian random field, p_target from a second field.  The FP32
    adjoint gradient (all 401 states stored) agrees with FP64 central finite
    differences (eps = 1e-3) along a smooth seeded direction to 1e-4, with
    the FP64 adjoint gradient to 1e-4, and costs at most 3x the forward."""
    from cfdarcov2_b200.workloads import adjoint_config, gaussian_random_field
    cfg = adjoint_config()
    n, steps, dt = cfg["n"], cfg["steps"], cfg["dt"]
    m = cfdb.Mesh.structured(ctx, n, n, n, 1 / n, 1 / n, 1 / n)
    q0_64 = dev(cfg["q0"], torch.float64)
    # p_target: forward run with the second field
    tgt = torch.empty(m.n, dtype=torch.float64, device=DEV)
    a, b = q0_64.clone(), torch.empty_like(q0_64)
    fin = ctx.wave_run(m, a, b, dt, steps, c=dev(cfg["c_true"], torch.float64), speed_mode=1, path=cfdb.PLAIN)
    tgt.copy_(fin[: m.n])
    c64 = dev(cfg["c"], torch.float64)
    g_c = torch.empty(m.n, device=DEV)
    g_p = torch.empty(m.n, device=DEV)
    J32, st = ctx.wave_gradient(m, q0_64.float(), c64.float(), tgt.float(), steps, dt, steps, g_c, g_p,
                                path=cfdb.FUSED)
    assert st.reverse_ms <= 3.0 * st.forward_ms, (st.forward_ms, st.reverse_ms)
    d = gaussian_random_field(n, corr=0.1, seed=9)
    d = dev(d / np.abs(d).max(), torch.float64)
    eps = 1e-3
    Jp = ctx.wave_objective(m, q0_64, c64 + eps * d, tgt, steps, dt, path=cfdb.PLAIN)
    Jm = ctx.wave_objective(m, q0_64, c64 - eps * d, tgt, steps, dt, path=cfdb.PLAIN)
    fd = (Jp - Jm) / (2 * eps)
    adj = float(torch.dot(g_c.double(), d))
    assert abs(adj - fd) <= 1e-4 * abs(fd), (adj, fd)
    g64 = torch.empty(m.n, dtype=torch.float64, device=DEV)
    gp64 = torch.empty(m.n, dtype=torch.float64, device=DEV)
    J64, _ = ctx.wave_gradient(m, q0_64, c64, tgt, steps, dt, steps, g64, gp64, path=cfdb.PLAIN)
    assert rel_l2(g_c.cpu().numpy(), g64.cpu().numpy()) <= 1e-4
    assert rel_l2(g_p.cpu().numpy(), gp64.cpu().numpy()) <= 1e-4
    assert J32 == pytest.approx(J64, rel=1e-4)
