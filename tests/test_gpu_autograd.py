"""The wave adjoint behind a torch.autograd.Function, as a PyTorch caller of
the inverse problem would bind it (test harness only; the library has no
torch dependency).

J(c, p0) = 1/2 ||p_T - p_target||^2 after T forward-Euler steps of the
first-order acoustic system (the d1t update of src/fvm3d.cpp:675-708 applied
to p, u, v, w with Rusanov fluxes), started from q0 = [p0 | 0 | 0 | 0].
forward() runs the forward sweep only (cfdb_wave_objective); backward()
runs the checkpointed forward + reverse sweep (cfdb_wave_gradient) and
returns dJ/dc and dJ/dp0 scaled by the incoming gradient."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


class WaveObjective(torch.autograd.Function):
    @staticmethod
    def forward(fctx, c, p0, lib_ctx, mesh, target, steps, dt, snapshots, path):
        n = mesh.n
        q0 = torch.zeros(4 * n, dtype=p0.dtype, device=p0.device)
        q0[:n] = p0.detach()
        J = lib_ctx.wave_objective(mesh, q0, c.detach().contiguous(), target, steps, dt, path=path)
        fctx.save_for_backward(c, q0)
        fctx.args = (lib_ctx, mesh, target, steps, dt, snapshots, path)
        return torch.tensor(J, dtype=p0.dtype, device=p0.device)

    @staticmethod
    def backward(fctx, gJ):
        c, q0 = fctx.saved_tensors
        lib_ctx, mesh, target, steps, dt, snapshots, path = fctx.args
        g_c = torch.empty(mesh.n, dtype=c.dtype, device=c.device)
        g_p = torch.empty(mesh.n, dtype=c.dtype, device=c.device)
        lib_ctx.wave_gradient(mesh, q0, c.detach().contiguous(), target, steps, dt, snapshots, g_c, g_p, path=path)
        return gJ * g_c, gJ * g_p, None, None, None, None, None, None, None


def objective(c, p0, lib_ctx, mesh, target, steps, dt, snapshots, path):
    return WaveObjective.apply(c, p0, lib_ctx, mesh, target, steps, dt, snapshots, path)


def test_gradcheck_fp64_plain(cfdb, ctx):
    """torch.autograd.gradcheck (central differences of the forward against
    the adjoint's Jacobian row) on a 5^3 mesh, 6 steps, 2 checkpoint slots."""
    n, steps = 5, 6
    m = cfdb.Mesh.structured(ctx, n, n, n, 1 / n, 1 / n, 1 / n)
    rng = np.random.default_rng(21)
    c = torch.tensor(np.exp(0.2 * rng.standard_normal(m.n)), dtype=torch.float64, device=DEV, requires_grad=True)
    p0 = torch.tensor(rng.standard_normal(m.n), dtype=torch.float64, device=DEV, requires_grad=True)
    target = torch.tensor(rng.standard_normal(m.n) * 0.1, dtype=torch.float64, device=DEV)
    dt = m.wave_dt(0.4, c=c.detach().cpu().numpy() * 1.2)
    assert torch.autograd.gradcheck(
        lambda cc, pp: objective(cc, pp, ctx, m, target, steps, dt, 2, cfdb.PLAIN), (c, p0),
        eps=1e-6, atol=1e-8, rtol=1e-6)


def test_backward_matches_library_gradient(cfdb, ctx):
    """J.backward() leaves exactly cfdb_wave_gradient's arrays in .grad, for
    the FP32 fused path and any checkpoint count."""
    n, steps = 16, 20
    m = cfdb.Mesh.structured(ctx, n, n, n, 1 / n, 1 / n, 1 / n)
    rng = np.random.default_rng(4)
    c = torch.tensor(np.exp(0.2 * rng.standard_normal(m.n)), dtype=torch.float32, device=DEV, requires_grad=True)
    p0 = torch.tensor(rng.standard_normal(m.n), dtype=torch.float32, device=DEV, requires_grad=True)
    target = torch.tensor(rng.standard_normal(m.n) * 0.1, dtype=torch.float32, device=DEV)
    dt = m.wave_dt(0.4, c=c.detach().cpu().numpy() * 1.2)
    J = objective(c, p0, ctx, m, target, steps, dt, 3, cfdb.FUSED)
    J.backward()
    q0 = torch.zeros(4 * m.n, device=DEV)
    q0[: m.n] = p0.detach()
    g_c, g_p = torch.empty(m.n, device=DEV), torch.empty(m.n, device=DEV)
    Jl, _ = ctx.wave_gradient(m, q0, c.detach(), target, steps, dt, steps, g_c, g_p, path=cfdb.FUSED)
    assert float(J) == pytest.approx(Jl, rel=1e-6)
    assert torch.equal(c.grad, g_c) and torch.equal(p0.grad, g_p)


def test_full_size_gradients_vs_central_fd(cfdb, ctx):
    """The adjoint workload at full size (128^3, 400 steps, c = exp(0.2 g),
    g a seeded Gaussian random field; p_target from a forward run with a
    second field).  Both gradients of the FP32 autograd backward agree with
    FP64 central differences (eps = 1e-3) along seeded smooth directions to
    1e-4: dJ/dc, and dJ/dp0 (J is quadratic in p0, so its central difference
    is exact up to round-off)."""
    from cfdarcov2_b200.workloads import adjoint_config, gaussian_random_field
    cfg = adjoint_config()
    n, steps, dt = cfg["n"], cfg["steps"], cfg["dt"]
    m = cfdb.Mesh.structured(ctx, n, n, n, 1 / n, 1 / n, 1 / n)
    q0_64 = torch.tensor(cfg["q0"], dtype=torch.float64, device=DEV)
    a, b = q0_64.clone(), torch.empty_like(q0_64)
    fin = ctx.wave_run(m, a, b, dt, steps, c=torch.tensor(cfg["c_true"], dtype=torch.float64, device=DEV),
                       speed_mode=1, path=cfdb.PLAIN)
    tgt64 = fin[: m.n].clone()
    c64 = torch.tensor(cfg["c"], dtype=torch.float64, device=DEV)
    p64 = q0_64[: m.n].clone()

    c = c64.float().requires_grad_(True)
    p0 = p64.float().requires_grad_(True)
    J = objective(c, p0, ctx, m, tgt64.float(), steps, dt, steps, cfdb.FUSED)
    J.backward()

    eps = 1e-3
    for seed, grad, which in ((9, c.grad, "c"), (10, p0.grad, "p0")):
        d = gaussian_random_field(n, corr=0.1, seed=seed)
        d = torch.tensor(d / np.abs(d).max(), dtype=torch.float64, device=DEV)

        def J64(delta):
            cc, pp = (c64 + delta, p64) if which == "c" else (c64, p64 + delta)
            return float(objective(cc, pp, ctx, m, tgt64, steps, dt, steps, cfdb.PLAIN))
        fd = (J64(eps * d) - J64(-eps * d)) / (2 * eps)
        adj = float(torch.dot(grad.double(), d))
        assert abs(adj - fd) <= 1e-4 * abs(fd), (which, adj, fd)
