"""GPU parity of the plain operator layer and the heat / wave time steps
against the CPU oracle, through the C ABI.

Bars: FP64 plain path bit-identical to the FP64 oracle (the north-star bar
is 1e-12 relative; identical operation order makes it exact); FP32 plain
path bit-identical to the FP32 oracle on power-of-two uniform meshes; FP32
fused path within L2 relative error 1e-5 of the FP64 oracle."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import rel_l2, rel_linf

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def dev(a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


MESHES = [
    dict(shape=(5, 6, 7), spacing=(0.2, 1 / 6, 1 / 7), verts=None),
    dict(shape=(8, 8, 8), spacing=(1 / 8, 1 / 8, 1 / 8), verts=None),
    dict(shape=(6, 6, 6), spacing=(1 / 6, 1 / 6, 1 / 6), verts="jitter"),
]


def make_pair(cfdb, oracle, ctx, spec, np_dtype):
    from cfdarcov2_b200.workloads import jittered_vertices
    shape, spacing = spec["shape"], spec["spacing"]
    if spec["verts"] == "jitter":
        V = jittered_vertices(shape[0], seed=2)
        return (cfdb.Mesh.from_vertices(ctx, *shape, *spacing, V),
                oracle.Mesh(*shape, *spacing, vertices=V, dtype=np_dtype))
    return cfdb.Mesh.structured(ctx, *shape, *spacing), oracle.Mesh(*shape, *spacing, dtype=np_dtype)


@pytest.mark.parametrize("spec", MESHES + [dict(shape=(7, 5, 9), spacing=(1 / 13, 0.3, 1 / 7), verts=None)],
                         ids=["aniso", "cube8", "jitter6", "odd"])
def test_device_built_geometry_equals_host_builder(cfdb, ctx, spec):
    """The face arrays are built on the device from the same formulas as the
    host builder: each FP32 array equals the host double rounded to float,
    and the neighbour ids match."""
    from cfdarcov2_b200.workloads import jittered_vertices
    shape, spacing = spec["shape"], spec["spacing"]
    if spec["verts"] == "jitter":
        m = cfdb.Mesh.from_vertices(ctx, *shape, *spacing, jittered_vertices(shape[0], seed=2))
    else:
        m = cfdb.Mesh.structured(ctx, *shape, *spacing)
    got = m.plain_geometry()
    cap = cfdb.capi
    for which, key in [(cap.GEOM_NORMAL, "normal"), (cap.GEOM_NORMAL_ALT, "normal_alt"), (cap.GEOM_AREA, "area"),
                       (cap.GEOM_ALPHA_D, "alpha"), (cap.GEOM_LEN_C2F, "len"), (cap.GEOM_VOLUME, "volume")]:
        assert np.array_equal(got[key], m.geometry(which).astype(np.float32)), key
    ids, _ = m.ids()
    assert np.array_equal(got["ids"].astype(np.int64), ids)


@pytest.mark.parametrize("shape,spacing", [((8, 8, 8), (1.0, 1.0, 1.0)), ((6, 5, 4), (0.25, 0.5, 2.0)),
                                           ((7, 5, 9), (1 / 13, 0.3, 1 / 7)), ((1, 4, 4), (1.0, 1.0, 1.0))])
def test_lattice_constants_agree_with_face_arrays(cfdb, ctx, shape, spacing):
    """cfdb_mesh_lattice_geometry says exact exactly when every cell's FP32
    face arrays equal the per-slot constants (alpha and len split by wall)."""
    m = cfdb.Mesh.structured(ctx, *shape, *spacing)
    exact, c = m.lattice_geometry()
    g = m.plain_geometry()
    nx, ny, nz = shape
    n = m.n
    x, y, z = (a.ravel() for a in np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"))
    wall = np.stack([z == 0, z == nz - 1, y == 0, y == ny - 1, x == 0, x == nx - 1]).astype(int)  # (6, n)
    f = np.arange(6)[:, None]
    bits = lambda a: np.asarray(a, np.float32).view(np.uint32)
    expect = {
        "normal": np.concatenate([np.broadcast_to(c["normal"][d * 6:d * 6 + 6, None], (6, n)).ravel() for d in range(3)]),
        "normal_alt": np.concatenate([np.broadcast_to(c["normal_alt"][d * 6:d * 6 + 6, None], (6, n)).ravel()
                                      for d in range(3)]),
        "area": np.broadcast_to(c["area"][:, None], (6, n)).ravel(),
        "alpha": c["alpha"][wall * 6 + f].ravel(),
        "len": c["len"][wall * 6 + f].ravel(),
        "volume": np.full(n, c["volume"], np.float32),
    }
    step = np.array([-1, 1, -nz, nz, -ny * nz, ny * nz])[:, None]
    i = np.arange(n)[None, :]
    ids = np.where(wall == 1, i, i + step).ravel()
    matches = all(np.array_equal(bits(g[k]), bits(v)) for k, v in expect.items()) and np.array_equal(g["ids"], ids)
    assert exact == matches
    if spacing == (1.0, 1.0, 1.0):
        assert exact


def test_lattice_check_rejects_vertex_meshes(cfdb, ctx):
    from cfdarcov2_b200.workloads import jittered_vertices
    m = cfdb.Mesh.from_vertices(ctx, 6, 6, 6, 1 / 6, 1 / 6, 1 / 6, jittered_vertices(6, seed=2))
    assert not m.lattice_geometry()[0]


@pytest.mark.parametrize("spec", MESHES, ids=["aniso", "cube8", "jitter6"])
@pytest.mark.parametrize("op", ["grad", "lapl", "stab"])
@pytest.mark.parametrize("mask", [7, 1, 6])
def test_plain_operators_fp64_bitwise(cfdb, oracle, ctx, spec, op, mask):
    m, o = make_pair(cfdb, oracle, ctx, spec, np.float64)
    rng = np.random.default_rng(7)
    phi = rng.standard_normal(m.n)
    got = host(getattr(ctx, op)(m, dev(phi, torch.float64), mask=mask))
    ref = getattr(o, op)(phi, mask)
    assert np.array_equal(got, ref), np.abs(got - ref).max()


@pytest.mark.parametrize("op", ["grad", "lapl", "stab"])
def test_plain_operators_fp32_bitwise_on_pow2_mesh(cfdb, oracle, ctx, op):
    m, o = make_pair(cfdb, oracle, ctx, MESHES[1], np.float32)
    rng = np.random.default_rng(8)
    phi = rng.standard_normal(m.n).astype(np.float32)
    got = host(getattr(ctx, op)(m, dev(phi, torch.float32)))
    ref = getattr(o, op)(phi)
    assert np.array_equal(got, ref), np.abs(got - ref).max()


def test_elementwise_and_time_operators(cfdb, ctx):
    cap = cfdb.capi
    rng = np.random.default_rng(9)
    for tdt, ndt in [(torch.float64, np.float64), (torch.float32, np.float32)]:
        a = rng.standard_normal(1000).astype(ndt)
        b = (rng.uniform(0.5, 2, 1000)).astype(ndt)
        ta, tb = dev(a, tdt), dev(b, tdt)
        assert np.array_equal(host(ctx.binary(cap.OP_ADD, ta, tb)), a + b)
        assert np.array_equal(host(ctx.binary(cap.OP_SUB, ta, tb)), a - b)
        assert np.array_equal(host(ctx.binary(cap.OP_MUL, ta, tb)), a * b)
        assert np.array_equal(host(ctx.binary(cap.OP_DIV, ta, tb)), a / b)
        s = ndt(0.37)
        assert np.array_equal(host(ctx.scalar(cap.OP_MUL, ta, float(s))), a * s)
        assert np.array_equal(host(ctx.scalar(cap.OP_RSUB, ta, float(s))), s - a)
        assert np.array_equal(host(ctx.scalar(cap.OP_RDIV, tb, float(s))), s / b)
        assert np.array_equal(host(ctx.neg(ta)), -a)
        assert np.all(host(ctx.fill(torch.empty_like(ta), 2.5)) == 2.5)
        dt = ndt(0.01)
        assert np.array_equal(host(ctx.d1t(ta, tb, float(dt))), dt * a + b)
        c = rng.standard_normal(1000).astype(ndt)
        tc = dev(c, tdt)
        assert np.array_equal(host(ctx.d2t(ta, tb, tc, float(dt), 1)), (dt * dt * a + ndt(2) * b) - c)
        assert np.array_equal(host(ctx.d2t(ta, tb, None, float(dt), 0)), dt * a + b)


def test_boundary_copy_and_cfl(cfdb, oracle, ctx):
    m = cfdb.Mesh.structured(ctx, 6, 5, 4, 0.1, 0.2, 0.3)
    o = oracle.Mesh(6, 5, 4, 0.1, 0.2, 0.3)
    rng = np.random.default_rng(10)
    arr, cp = rng.standard_normal(m.n), rng.standard_normal(m.n)
    isb = o.geometry()["is_boundary"]
    got = host(ctx.boundary_copy(m, dev(arr, torch.float64), dev(cp, torch.float64)))
    assert np.array_equal(got, arr * (1 - isb) + cp * isb)
    # the in-place boundary-only form gives the same values (finite, no -0 here)
    for shape in [(6, 5, 4), (1, 3, 4), (2, 2, 2), (7, 1, 1)]:
        mb = cfdb.Mesh.structured(ctx, *shape, 0.1, 0.2, 0.3)
        ob = oracle.Mesh(*shape, 0.1, 0.2, 0.3)
        a, c = rng.standard_normal(mb.n).astype(np.float32), rng.standard_normal(mb.n).astype(np.float32)
        b = ob.geometry()["is_boundary"].astype(np.float32)
        ta = dev(a, torch.float32)
        ctx.boundary_set(mb, ta, dev(c, torch.float32))
        assert np.array_equal(host(ta), a * (1 - b) + c * b), shape
    p, rho = rng.uniform(0.5, 2, m.n), rng.uniform(0.5, 2, m.n)
    u, v, w = rng.standard_normal((3, m.n))
    d = lambda x: dev(x, torch.float64)  # noqa: E731
    assert ctx.cfl_dt(m, 0.4, 5 / 3, d(p), d(rho), d(u), d(v), d(w)) == o.cfl_reference(0.4, 5 / 3, p, rho, u, v, w)
    assert ctx.cfl_dt(m, 0.4, 5 / 3, d(p), d(rho), d(u)) == o.cfl_reference(0.4, 5 / 3, p, rho, u)


def test_total_fp64(cfdb, oracle, ctx):
    m = cfdb.Mesh.structured(ctx, 32, 16, 8, 1 / 32, 1 / 16, 1 / 8)
    o = oracle.Mesh(32, 16, 8, 1 / 32, 1 / 16, 1 / 8)
    rng = np.random.default_rng(11)
    f = rng.uniform(0, 1, m.n)
    assert ctx.total_fp64(m, dev(f, torch.float64)) == pytest.approx(o.total(f), rel=1e-14)
    f32 = f.astype(np.float32)
    assert ctx.total_fp64(m, dev(f32, torch.float32)) == pytest.approx(o.total(f32.astype(np.float64)), rel=1e-14)


def run_steps(step, a, b, steps):
    for _ in range(steps):
        step(a, b)
        a, b = b, a
    return a


def test_heat_plain_fp64_matches_oracle_bitwise_config1(cfdb, oracle, ctx):
    """The heat workload (64^3, k = 0.01, dt = 0.1 dx^2/k, 200 steps) on the
    FP64 plain path is bit-identical to the FP64 oracle (bar: 1e-12 rel)."""
    from cfdarcov2_b200.workloads import heat_config
    cfg = heat_config()
    n = cfg["n"]
    m = cfdb.Mesh.structured(ctx, n, n, n, cfg["dx"], cfg["dx"], cfg["dx"])
    o = oracle.Mesh(n, n, n, cfg["dx"], cfg["dx"], cfg["dx"])
    a = dev(cfg["T0"], torch.float64)
    b = torch.empty_like(a)
    out = run_steps(lambda x, y: ctx.heat_step(m, x, y, cfg["k"], cfg["dt"], path=cfdb.PLAIN), a, b, cfg["steps"])
    ref = o.heat_solve(cfg["T0"], cfg["k"], cfg["dt"], cfg["steps"])
    got = host(out)
    assert rel_linf(got, ref) <= 1e-12
    assert np.array_equal(got, ref)


def test_heat_fused_fp32_within_tolerance(cfdb, oracle, ctx):
    from cfdarcov2_b200.workloads import heat_config
    cfg = heat_config(n=32, steps=100)
    n = cfg["n"]
    m = cfdb.Mesh.structured(ctx, n, n, n, cfg["dx"], cfg["dx"], cfg["dx"])
    o = oracle.Mesh(n, n, n, cfg["dx"], cfg["dx"], cfg["dx"])
    a = dev(cfg["T0"], torch.float32)
    b = torch.empty_like(a)
    out = run_steps(lambda x, y: ctx.heat_step(m, x, y, cfg["k"], cfg["dt"], path=cfdb.FUSED), a, b, cfg["steps"])
    ref = o.heat_solve(cfg["T0"], cfg["k"], cfg["dt"], cfg["steps"])
    assert rel_l2(host(out), ref) <= 1e-5
    assert rel_linf(host(out), ref) <= 1e-5


@pytest.mark.parametrize("shape", [(12, 8, 16), (9, 5, 4), (3, 17, 36), (20, 3, 132)])
def test_heat_fused_edge_shapes(cfdb, oracle, ctx, shape):
    """Partial tiles in y and z, thin meshes, chunk boundaries in x."""
    nx, ny, nz = shape
    m = cfdb.Mesh.structured(ctx, nx, ny, nz, 1 / nx, 1 / ny, 1 / nz)
    o = oracle.Mesh(nx, ny, nz, 1 / nx, 1 / ny, 1 / nz)
    rng = np.random.default_rng(12)
    T0 = rng.uniform(size=m.n)
    dt = 0.1 / (nx * nx + ny * ny + nz * nz)
    a = dev(T0, torch.float32)
    b = torch.empty_like(a)
    out = run_steps(lambda x, y: ctx.heat_step(m, x, y, 1.0, dt, path=cfdb.FUSED), a, b, 7)
    ref = o.heat_solve(T0, 1.0, dt, 7)
    assert rel_linf(host(out), ref) <= 3e-6


@pytest.mark.parametrize("shape", [(16, 12, 8), (9, 5, 4), (3, 7, 132), (1, 1, 8)])
def test_heat_step_fixed_equals_step_then_boundary_set(cfdb, ctx, shape):
    """cfdb_heat_step_fixed (the boundary copy inside the fused step) gives
    the bits of cfdb_heat_step followed by cfdb_op_boundary_set; the surface
    cells hold the fixed values, the interior the heat update."""
    nx, ny, nz = shape
    m = cfdb.Mesh.structured(ctx, nx, ny, nz, 1 / nx, 1 / ny, 1 / nz)
    g = torch.Generator(device="cpu").manual_seed(11)
    T = torch.rand(m.n, generator=g).to(DEV)
    fixed = torch.rand(m.n, generator=g).to(DEV) + 2.0
    a, b = torch.empty_like(T), torch.empty_like(T)
    ctx.heat_step(m, T, a, 0.7, 1e-6, path=cfdb.FUSED)  # stable for every shape here (k dt / h^2 < 1/6)
    ctx.boundary_set(m, a, fixed)
    ctx.heat_step_fixed(m, T, b, 0.7, 1e-6, fixed)
    assert torch.equal(a, b)
    x, y, z = torch.meshgrid(torch.arange(nx), torch.arange(ny), torch.arange(nz), indexing="ij")
    surf = ((x == 0) | (x == nx - 1) | (y == 0) | (y == ny - 1) | (z == 0) | (z == nz - 1)).reshape(-1).to(DEV)
    assert torch.equal(b[surf], fixed[surf])
    assert not torch.any(b[~surf] >= 2.0)


@pytest.mark.parametrize("count,dtype", [(3, torch.float32), (17, torch.float32), (2, torch.float64)])
def test_boundary_set_many_equals_one_by_one(cfdb, ctx, count, dtype):
    """cfdb_op_boundary_set_many (one launch per 16 fields) writes what
    cfdb_op_boundary_set writes field by field, and nothing else."""
    m = cfdb.Mesh.structured(ctx, 9, 6, 8, 1 / 9, 1 / 6, 1 / 8)
    g = torch.Generator(device="cpu").manual_seed(2)
    fields = [torch.rand(m.n, generator=g, dtype=dtype).to(DEV) for _ in range(count)]
    values = [torch.rand(m.n, generator=g, dtype=dtype).to(DEV) for _ in range(count)]
    one = [f.clone() for f in fields]
    for f, v in zip(one, values):
        ctx.boundary_set(m, f, v)
    ctx.boundary_set_many(m, fields, values)
    for a, b in zip(fields, one):
        assert torch.equal(a, b)
    ctx.boundary_set_many(m, [], [])  # nothing to do


def test_heat_step_fixed_rejects_bad_arguments(cfdb, ctx):
    m = cfdb.Mesh.structured(ctx, 8, 8, 8, 1 / 8, 1 / 8, 1 / 8)
    T, Tn, fx = (torch.zeros(m.n, device=DEV) for _ in range(3))
    for args, code in (((T, Tn, None), cfdb.capi.EINVAL), ((T, Tn, Tn), cfdb.capi.EINVAL),
                       ((T, T, fx), cfdb.capi.EINVAL),
                       ((T.double(), Tn.double(), fx.double()), cfdb.capi.EUNSUPPORTED)):
        with pytest.raises(cfdb.CfdbError) as e:
            ctx.heat_step_fixed(m, args[0], args[1], 1.0, 1e-4, args[2])
        assert e.value.code == code
    m6 = cfdb.Mesh.structured(ctx, 4, 4, 6, 0.25, 0.25, 1 / 6)
    a, b, c = (torch.zeros(m6.n, device=DEV) for _ in range(3))
    with pytest.raises(cfdb.CfdbError) as e:
        ctx.heat_step_fixed(m6, a, b, 1.0, 1e-4, c)
    assert e.value.code == cfdb.capi.EUNSUPPORTED
    ctx.sync()


def test_fused_requires_nz_multiple_of_4(cfdb, ctx):
    m = cfdb.Mesh.structured(ctx, 4, 4, 6, 0.25, 0.25, 1 / 6)
    a = torch.zeros(m.n, device=DEV)
    b = torch.zeros(m.n, device=DEV)
    with pytest.raises(cfdb.CfdbError) as e:
        ctx.heat_step(m, a, b, 1.0, 0.001, path=cfdb.FUSED)
    assert e.value.code == cfdb.capi.EUNSUPPORTED
    ctx.heat_step(m, a, b, 1.0, 0.001, path=cfdb.PLAIN)  # the plain path serves any shape


@pytest.mark.parametrize("shape,spacing,masks,k", [((16, 12, 8), (1.0, 1.0, 1.0), [1, 2], 0.09),
                                                   ((10, 9, 12), (0.5, 0.25, 0.125), [7], 1.0),
                                                   ((8, 8, 16), (1 / 8, 1 / 8, 1 / 16), [4, 1, 2], 0.3),
                                                   ((5, 7, 4), (1.0, 2.0, 0.5), [3, 6], -1.5),
                                                   ((8, 6, 8), (1.0, 1.0, 3.0), [7], 0.5),
                                                   ((9, 4, 8), (1.0, 1.0, 1.0), [1, 2, 4], 0.25),
                                                   ((12, 8, 8), (1.0, 1.0, 1.0), [7], 0.7),
                                                   ((8, 8, 8), (1.0, 1.0, 1.0), [2, 1], 1.3),
                                                   ((16, 8, 8), (0.5, 0.5, 0.5), [1, 2], 0.2),
                                                   ((4, 3, 136), (1.0, 1.0, 1.0), [1, 2], 0.09)])
def test_d2t_fused_equals_operator_composition_bitwise(cfdb, ctx, shape, spacing, masks, k):
    """cfdb_d2t_step (one TMA pass) gives the bits of the operator kernels
    composed as the generated kernel of d2t(u) = k (L_m1(u) + L_m2(u) + ...)
    computes: Laplacians by direction mask, their sum left to right, times k,
    then the leapfrog update (first step: the d1t form).  Covers unit cells
    (products by one left out), power-of-two volumes (an exact 1/V) and
    V = 3 (a true division), each with the masks compiled in ([1, 2], [7],
    [1, 2, 4]) and read at run time; nz = 136 takes the 64-wide tiles."""
    m = cfdb.Mesh.structured(ctx, *shape, *spacing)
    assert m.lattice_geometry()[0]
    g = torch.Generator(device="cpu").manual_seed(5)
    u = torch.rand(m.n, generator=g).to(DEV)
    prev = torch.rand(m.n, generator=g).to(DEV)
    dt = torch.tensor(0.05, dtype=torch.float32, device=DEV)
    S = None
    for mk in masks:
        L = ctx.lapl(m, u, mask=mk)
        S = L if S is None else S + L
    R = torch.tensor(k, dtype=torch.float32, device=DEV) * S
    nxt = torch.empty_like(u)
    ctx.d2t_step(m, u, prev, nxt, k, masks, 0.05)
    assert torch.equal(nxt, (dt * dt * R + 2.0 * u) - prev)
    ctx.d2t_step(m, u, None, nxt, k, masks, 0.05, first_step=True)
    assert torch.equal(nxt, dt * R + u)


def test_d2t_fused_rejects_what_it_cannot_run(cfdb, ctx):
    m = cfdb.Mesh.structured(ctx, 8, 8, 8, 1.0, 1.0, 1.0)
    u, p, o = (torch.zeros(m.n, device=DEV) for _ in range(3))
    for masks in ([], [8], [1, 2, 4, 7]):
        with pytest.raises(cfdb.CfdbError) as e:
            ctx.d2t_step(m, u, p, o, 1.0, masks, 0.1)
        assert e.value.code == cfdb.capi.EINVAL
    with pytest.raises(cfdb.CfdbError) as e:
        ctx.d2t_step(m, u, p, u, 1.0, [7], 0.1)  # in place
    assert e.value.code == cfdb.capi.EINVAL
    with pytest.raises(cfdb.CfdbError) as e:
        ctx.d2t_step(m, u.double(), p.double(), o.double(), 1.0, [7], 0.1)
    assert e.value.code == cfdb.capi.EUNSUPPORTED
    m6 = cfdb.Mesh.structured(ctx, 4, 4, 6, 1.0, 1.0, 1.0)  # rows of 6 floats: no TMA sweep
    a, b = torch.zeros(m6.n, device=DEV), torch.zeros(m6.n, device=DEV)
    with pytest.raises(cfdb.CfdbError) as e:
        ctx.d2t_step(m6, a, None, b, 1.0, [7], 0.1, first_step=True)
    assert e.value.code == cfdb.capi.EUNSUPPORTED
    mr = cfdb.Mesh.structured(ctx, 7, 5, 8, 1 / 13, 0.3, 1 / 7)
    a, b = torch.zeros(mr.n, device=DEV), torch.zeros(mr.n, device=DEV)
    if not mr.lattice_geometry()[0]:  # geometry constants that differ between cells
        with pytest.raises(cfdb.CfdbError) as e:
            ctx.d2t_step(mr, a, None, b, 1.0, [7], 0.1, first_step=True)
        assert e.value.code == cfdb.capi.EUNSUPPORTED and "exact lattice" in str(e.value)
    ctx.sync()


@pytest.mark.parametrize("spec", MESHES, ids=["aniso", "cube8", "jitter6"])
@pytest.mark.parametrize("mode", [0, 1])
def test_wave_plain_fp64_bitwise(cfdb, oracle, ctx, spec, mode):
    m, o = make_pair(cfdb, oracle, ctx, spec, np.float64)
    rng = np.random.default_rng(13)
    q0 = rng.standard_normal(4 * m.n)
    c = np.exp(0.2 * rng.standard_normal(m.n))
    dt = o.wave_dt(0.4, c=c)
    a = dev(q0, torch.float64)
    b = torch.empty_like(a)
    tc = dev(c, torch.float64)
    out = run_steps(lambda x, y: ctx.wave_step(m, x, y, dt, c=tc, speed_mode=mode, path=cfdb.PLAIN), a, b, 6)
    ref = o.wave_solve(q0, dt, 6, c=c, speed_mode=mode)
    assert np.array_equal(host(out), ref)


@pytest.mark.parametrize("shape", [(16, 16, 16), (10, 7, 20), (24, 9, 132)])
@pytest.mark.parametrize("cfield", [False, True])
def test_wave_fused_fp32_vs_fp64_oracle(cfdb, oracle, ctx, shape, cfield):
    nx, ny, nz = shape
    m = cfdb.Mesh.structured(ctx, nx, ny, nz, 1 / nx, 1 / ny, 1 / nz)
    o = oracle.Mesh(nx, ny, nz, 1 / nx, 1 / ny, 1 / nz)
    rng = np.random.default_rng(14)
    q0 = rng.standard_normal(4 * m.n)
    c = np.exp(0.2 * rng.standard_normal(m.n)) if cfield else None
    mode = 1 if cfield else 0
    dt = o.wave_dt(0.4, c=c)
    a = dev(q0, torch.float32)
    b = torch.empty_like(a)
    tc = None if c is None else dev(c, torch.float32)
    out = run_steps(lambda x, y: ctx.wave_step(m, x, y, dt, c=tc, speed_mode=mode, path=cfdb.FUSED), a, b, 10)
    ref = o.wave_solve(q0, dt, 10, c=c, speed_mode=mode)
    assert rel_l2(host(out), ref) <= 1e-5


def test_wave_fused_distorted_vs_fp64_oracle(cfdb, oracle, ctx):
    from cfdarcov2_b200.workloads import jittered_vertices, wave_state
    n = 16
    V = jittered_vertices(n, seed=2)
    m = cfdb.Mesh.from_vertices(ctx, n, n, n, 1 / n, 1 / n, 1 / n, V)
    o = oracle.Mesh(n, n, n, 1 / n, 1 / n, 1 / n, vertices=V)
    q0 = wave_state(n, sigma=0.1)
    dt = o.wave_dt(0.4)
    a = dev(q0, torch.float32)
    b = torch.empty_like(a)
    out = run_steps(lambda x, y: ctx.wave_step(m, x, y, dt, path=cfdb.FUSED), a, b, 20)
    ref = o.wave_solve(q0, dt, 20)
    assert rel_l2(host(out), ref) <= 1e-5


def _jittered_box(nx, ny, nz, seed):
    """(nx+1)(ny+1)(nz+1) vertices of the unit box's lattice, interior ones
    jittered by U(-0.2, 0.2) of the local spacing (walls stay planar)."""
    rng = np.random.default_rng(seed)
    g = np.meshgrid(np.arange(nx + 1) / nx, np.arange(ny + 1) / ny, np.arange(nz + 1) / nz, indexing="ij")
    V = np.stack(g, axis=-1)
    J = rng.uniform(-0.2, 0.2, V.shape) * np.array([1 / nx, 1 / ny, 1 / nz])
    inner = np.zeros(V.shape[:3], bool)
    inner[1:-1, 1:-1, 1:-1] = True
    return (V + J * inner[..., None]).reshape(-1, 3)


# z extents on both sides of the 32/64-wide tile choice of the face sweep,
# partial y and z tiles, x shorter than the chunk count, meshes one cell thick
# in x or y and the smallest nz; nz = 13 and a c field take the gather form
@pytest.mark.parametrize("shape,cfield", [((20, 12, 24), False), ((9, 7, 68), False), ((6, 70, 8), False),
                                          ((11, 9, 132), False), ((1, 5, 8), False), ((3, 1, 12), False),
                                          ((2, 3, 4), False), ((7, 9, 13), False), ((10, 6, 12), True)])
def test_wave_fused_distorted_ragged_vs_fp64_oracle(cfdb, oracle, ctx, shape, cfield):
    nx, ny, nz = shape
    V = _jittered_box(nx, ny, nz, seed=5)
    m = cfdb.Mesh.from_vertices(ctx, nx, ny, nz, 1 / nx, 1 / ny, 1 / nz, V)
    o = oracle.Mesh(nx, ny, nz, 1 / nx, 1 / ny, 1 / nz, vertices=V)
    rng = np.random.default_rng(6)
    q0 = 0.1 * rng.standard_normal(4 * m.n)
    c = np.exp(0.2 * rng.standard_normal(m.n)) if cfield else None
    mode = 1 if cfield else 0
    dt = o.wave_dt(0.4, c=c)
    a = dev(q0, torch.float32)
    b = torch.empty_like(a)
    tc = None if c is None else dev(c, torch.float32)
    out = run_steps(lambda x, y: ctx.wave_step(m, x, y, dt, c=tc, speed_mode=mode, path=cfdb.FUSED), a, b, 12)
    ref = o.wave_solve(q0, dt, 12, c=c, speed_mode=mode)
    assert rel_l2(host(out), ref) <= 1e-5
    assert rel_linf(host(out), ref) <= 1e-5


def test_wave_config2_fused_fp32_vs_fp64_plain_full_size(cfdb, ctx):
    """The wave workload at full size (128^3, 500 steps): FP32 fused vs the
    FP64 plain GPU path (bit-identical to the FP64 oracle on the small cases
    above), L2 relative error <= 1e-5, and the pressure integral conserved."""
    from cfdarcov2_b200.workloads import wave_config
    cfg = wave_config()
    n = cfg["n"]
    m = cfdb.Mesh.structured(ctx, n, n, n, cfg["dx"], cfg["dx"], cfg["dx"])
    a64 = dev(cfg["q0"], torch.float64)
    b64 = torch.empty_like(a64)
    ref = run_steps(lambda x, y: ctx.wave_step(m, x, y, cfg["dt"], c_const=cfg["c"], path=cfdb.PLAIN), a64, b64,
                    cfg["steps"])
    a32 = dev(cfg["q0"], torch.float32)
    b32 = torch.empty_like(a32)
    got = run_steps(lambda x, y: ctx.wave_step(m, x, y, cfg["dt"], c_const=cfg["c"], path=cfdb.FUSED), a32, b32,
                    cfg["steps"])
    r, g = host(ref), host(got)
    assert rel_l2(g, r) <= 1e-5
    N = m.n
    p0 = cfg["q0"][:N].sum()
    assert abs(r[:N].sum() - p0) <= 1e-10 * p0


@pytest.mark.parametrize("path", ["plain", "fused"])
def test_graph_run_equals_eager_steps(cfdb, ctx, path):
    """cfdb_wave_run / cfdb_heat_run replaying a captured CUDA graph give the
    same bits as step-by-step launches, for odd and even step counts."""
    P = cfdb.FUSED if path == "fused" else cfdb.PLAIN
    n = 24
    m = cfdb.Mesh.structured(ctx, n, n, n, 1 / n, 1 / n, 1 / n)
    rng = np.random.default_rng(15)
    q0 = dev(rng.standard_normal(4 * m.n), torch.float32)
    dt = m.wave_dt(0.4)
    for steps in (1, 2, 7, 70, 131):
        a, b = q0.clone(), torch.empty_like(q0)
        ref = run_steps(lambda x, y: ctx.wave_step(m, x, y, dt, path=P), a, b, steps)
        a2, b2 = q0.clone(), torch.empty_like(q0)
        got = ctx.wave_run(m, a2, b2, dt, steps, path=P, use_graph=True)
        assert torch.equal(host_t(got), host_t(ref)), steps
    T0 = dev(rng.uniform(size=m.n), torch.float32)
    a, b = T0.clone(), torch.empty_like(T0)
    ref = run_steps(lambda x, y: ctx.heat_step(m, x, y, 0.1, 1e-4, path=P), a, b, 67)
    a2, b2 = T0.clone(), torch.empty_like(T0)
    got = ctx.heat_run(m, a2, b2, 0.1, 1e-4, 67, path=P)
    assert torch.equal(host_t(got), host_t(ref))


def host_t(t):
    torch.cuda.synchronize()
    return t.detach().cpu()


@pytest.mark.parametrize("path", ["plain", "fused"])
def test_launch_count_and_cached_graph_replay(cfdb, ctx, path):
    """cfdb_ctx_launch_count counts every kernel, graph replays included; a
    repeated run with the same mesh, buffers and parameters replays the
    cached graph (no second recording) and gives the same bits as the first
    run and as step-by-step launches."""
    P = cfdb.FUSED if path == "fused" else cfdb.PLAIN
    n = 32
    m = cfdb.Mesh.structured(ctx, n, n, n, 1 / n, 1 / n, 1 / n)
    q0 = dev(np.random.default_rng(21).standard_normal(4 * m.n), torch.float32)
    dt = m.wave_dt(0.4)
    a, b = q0.clone(), torch.empty_like(q0)
    ctx.wave_step(m, a, b, dt, path=P)  # one-time setup (plain geometry upload) outside the counts
    per_step = 1 if path == "fused" else None
    c0 = ctx.launch_count()
    ctx.wave_step(m, a, b, dt, path=P)
    one = ctx.launch_count() - c0
    if per_step is not None:
        assert one == per_step
    steps = 100
    outs = []
    for _ in range(2):
        a.copy_(q0)
        c0 = ctx.launch_count()
        outs.append(host_t(ctx.wave_run(m, a, b, dt, steps, path=P, use_graph=True)).clone())
        assert ctx.launch_count() - c0 == steps * one
    assert torch.equal(outs[0], outs[1])
    x, y = q0.clone(), torch.empty_like(q0)
    ref = run_steps(lambda s, d: ctx.wave_step(m, s, d, dt, path=P), x, y, steps)
    assert torch.equal(outs[0], host_t(ref))
