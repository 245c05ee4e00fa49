"""Compressible Euler (first-order Rusanov) through the C ABI: the FP64 plain
path is bit-identical to the FP64 oracle for a whole Sod run (device-side dt,
last step clipped onto t_end, FP64 totals per step); the FP32 fused path is
compared with the FP64 oracle and with the exact Riemann solution."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def sod(nx, ny, nz, lyz=None):
    from cfdarcov2_b200.workloads import sod_state
    lyz = lyz if lyz is not None else 0.125
    U0, (dx, dy, dz) = sod_state(nx, ny, nz, 1.0, lyz)
    return U0, dx, dy, dz


def run_gpu(cfdb, ctx, mesh, U0, dtype, path, t_end, check_every=16):
    tdt = torch.float64 if dtype == cfdb.F64 else torch.float32
    e = cfdb.Euler(ctx, mesh, dtype=dtype, path=path, gamma=1.4, cfl=0.4, t_end=t_end, max_steps=20000)
    a = torch.tensor(U0, dtype=tdt, device=DEV)
    b = torch.empty_like(a)
    e.begin(a)
    steps, in_b = e.run(a, b, check_every)
    t, s2, fin = e.status()
    out = (b if in_b else a).double().cpu().numpy()
    return out, steps, t, fin, e.totals()


def test_plain_fp64_bitwise_vs_oracle(cfdb, oracle, ctx):
    U0, dx, dy, dz = sod(64, 4, 4, 0.0625)
    m = cfdb.Mesh.structured(ctx, 64, 4, 4, dx, dy, dz)
    o = oracle.Mesh(64, 4, 4, dx, dy, dz)
    got, steps, t, fin, tot = run_gpu(cfdb, ctx, m, U0, cfdb.F64, cfdb.PLAIN, 0.2)
    ref, rsteps, rt, rtot = o.euler_solve(U0, 1.4, 0.4, 0.2)
    assert fin and steps == rsteps and t == rt == 0.2
    assert np.array_equal(got, ref)
    assert np.allclose(tot, rtot, rtol=1e-14, atol=0)


def test_plain_fp64_bitwise_on_vertex_mesh(cfdb, oracle, ctx):
    from cfdarcov2_b200.workloads import jittered_vertices
    n = 8
    V = jittered_vertices(n, amp=0.1, seed=3)
    m = cfdb.Mesh.from_vertices(ctx, n, n, n, 1 / n, 1 / n, 1 / n, V)
    o = oracle.Mesh(n, n, n, 1 / n, 1 / n, 1 / n, vertices=V)
    c = o.geometry()["center"].reshape(3, -1)
    rho = np.where(c[0] < 0.5, 1.0, 0.125)
    U0 = np.zeros(5 * m.n)
    U0[: m.n] = rho
    U0[4 * m.n:] = np.where(c[0] < 0.5, 1.0, 0.1) / 0.4
    got, steps, t, fin, tot = run_gpu(cfdb, ctx, m, U0, cfdb.F64, cfdb.PLAIN, 0.05)
    ref, rsteps, rt, rtot = o.euler_solve(U0, 1.4, 0.4, 0.05)
    assert steps == rsteps and np.array_equal(got, ref)


def test_fused_fp32_vs_fp64_oracle(cfdb, oracle, ctx):
    U0, dx, dy, dz = sod(128, 8, 8, 0.0625)
    m = cfdb.Mesh.structured(ctx, 128, 8, 8, dx, dy, dz)
    o = oracle.Mesh(128, 8, 8, dx, dy, dz)
    got, steps, t, fin, tot = run_gpu(cfdb, ctx, m, U0, cfdb.F32, cfdb.FUSED, 0.2)
    ref, rsteps, rt, rtot = o.euler_solve(U0, 1.4, 0.4, 0.2)
    assert fin and t == 0.2 and abs(steps - rsteps) <= 1
    assert rel_l2(got, ref) <= 1e-5
    # FP64 totals of the FP32 state: mass and energy conserved to round-off
    assert np.abs(tot[:, 0] - tot[0, 0]).max() <= 1e-6 * tot[0, 0]
    assert np.abs(tot[:, 1] - tot[0, 1]).max() <= 1e-6 * tot[0, 1]


def blast(X, Y, Z, seed=7):
    """A 3-D state with structure along every axis: an off-centre pressure
    and density bump plus a seeded smooth velocity field."""
    rng = np.random.default_rng(seed)
    x = (np.arange(X) + 0.5) / X
    y = (np.arange(Y) + 0.5) / Y
    z = (np.arange(Z) + 0.5) / Z
    gx, gy, gz = np.meshgrid(x, y, z, indexing="ij")
    r2 = (gx - 0.4) ** 2 + (gy - 0.55) ** 2 + (gz - 0.45) ** 2
    bump = np.exp(-r2 / 0.02)
    rho = 1.0 + 0.3 * bump
    p = 1.0 + 2.0 * bump
    k = rng.uniform(1, 3, size=(3, 3))
    ph = rng.uniform(0, 2 * np.pi, size=3)
    u = [0.2 * np.sin(2 * np.pi * (k[d, 0] * gx + k[d, 1] * gy + k[d, 2] * gz) + ph[d]) for d in range(3)]
    E = p / 0.4 + 0.5 * rho * (u[0] ** 2 + u[1] ** 2 + u[2] ** 2)
    return np.concatenate([rho.ravel(), (rho * u[0]).ravel(), (rho * u[1]).ravel(), (rho * u[2]).ravel(), E.ravel()])


@pytest.mark.parametrize("shape", [(24, 20, 36), (16, 9, 68), (12, 33, 8), (1, 6, 8), (9, 1, 12), (3, 5, 4)])
def test_fused_fp32_3d_vs_fp64_oracle(cfdb, oracle, ctx, shape):
    """Structure along x, y and z: exercises the face fluxes of every
    direction, the z faces between a thread's cells and across threads and
    tiles (32- and 64-wide z tiles, partial tiles), and every wall; meshes
    one cell thick in x or y have both walls of that axis on one cell, and
    nz = 4 is the smallest z extent of the fused path."""
    X, Y, Z = shape
    U0 = blast(X, Y, Z)
    m = cfdb.Mesh.structured(ctx, X, Y, Z, 1 / X, 1 / Y, 1 / Z)
    o = oracle.Mesh(X, Y, Z, 1 / X, 1 / Y, 1 / Z)
    got, steps, t, fin, tot = run_gpu(cfdb, ctx, m, U0, cfdb.F32, cfdb.FUSED, 0.05)
    ref, rsteps, rt, rtot = o.euler_solve(U0, 1.4, 0.4, 0.05)
    assert fin and abs(steps - rsteps) <= 1
    assert rel_l2(got, ref) <= 1e-5


def test_fused_full_size_sod_matches_exact_riemann(cfdb, ctx):
    """The Sod workload at full size (512 x 64 x 64 on [0,1] x [0,0.125]^2 to
    t = 0.2): the density profile is uniform across y/z (walls are reflective
    and the data is 1-D) and close to the exact Riemann solution."""
    from oracle import riemann
    U0, dx, dy, dz = sod(512, 64, 64)
    m = cfdb.Mesh.structured(ctx, 512, 64, 64, dx, dy, dz)
    got, steps, t, fin, tot = run_gpu(cfdb, ctx, m, U0, cfdb.F32, cfdb.FUSED, 0.2, check_every=64)
    assert fin and t == 0.2
    rho = got[: m.n].reshape(512, 64 * 64)
    assert np.abs(rho - rho[:, :1]).max() <= 1e-5
    xc = (np.arange(512) + 0.5) * dx
    ex = riemann.sample(xc, 0.2, 0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    assert np.mean(np.abs(rho[:, 0] - ex[0])) < 0.01
    assert np.abs(tot[:, 0] - tot[0, 0]).max() <= 1e-6 * tot[0, 0]


def test_fused_and_plain_fp32_agree(cfdb, ctx):
    U0, dx, dy, dz = sod(64, 8, 8, 0.125)
    m = cfdb.Mesh.structured(ctx, 64, 8, 8, dx, dy, dz)
    a, s1, *_ = run_gpu(cfdb, ctx, m, U0, cfdb.F32, cfdb.FUSED, 0.1)
    b, s2, *_ = run_gpu(cfdb, ctx, m, U0, cfdb.F32, cfdb.PLAIN, 0.1)
    assert abs(s1 - s2) <= 1 and rel_l2(a, b) <= 1e-5


def test_step_after_finish_is_a_noop_and_max_steps_bounds(cfdb, ctx):
    U0, dx, dy, dz = sod(32, 4, 4, 0.125)
    m = cfdb.Mesh.structured(ctx, 32, 4, 4, dx, dy, dz)
    e = cfdb.Euler(ctx, m, dtype=cfdb.F32, path=cfdb.FUSED, t_end=0.2, max_steps=5)
    a = torch.tensor(U0, dtype=torch.float32, device=DEV)
    b = torch.empty_like(a)
    e.begin(a)
    for k in range(12):
        (e.step(a, b) if k % 2 == 0 else e.step(b, a))
    t, steps, fin = e.status()
    assert steps == 5 and fin and t < 0.2
    assert e.totals().shape == (6, 2)


def test_euler_rejects_bad_arguments(cfdb, ctx):
    m = cfdb.Mesh.structured(ctx, 8, 8, 6, 0.1, 0.1, 0.1)
    with pytest.raises(cfdb.CfdbError) as ei:
        cfdb.Euler(ctx, m, dtype=cfdb.F32, path=cfdb.FUSED)
    assert ei.value.code == cfdb.capi.EUNSUPPORTED  # nz % 4 != 0 on the TMA path
    with pytest.raises(cfdb.CfdbError):
        cfdb.Euler(ctx, m, dtype=cfdb.F32, path=cfdb.PLAIN, gamma=1.0)
