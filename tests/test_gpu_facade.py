"""The drop-in C++ facade (include/cfdb/fvm3d.hpp) driven like the reference's
examples: the example program builds Mesh3D / Variable / DT /
EquationTemplate / Equation::evaluate, runs on the GPU through libcfdb, and
its result is compared with the CPU oracle run step by step."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "cfdarcov2_b200", "_lib", "fvm_example")


def run_example(tmp_path, mode, nx, ny, nz, steps, nfields=1):
    out = tmp_path / f"{mode}.bin"
    r = subprocess.run([EXE, mode, str(out), str(nx), str(ny), str(nz), str(steps)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    data = np.fromfile(out, dtype=np.float32).astype(np.float64)
    return data.reshape(nfields, -1), r.stdout


def gaussian(m, c, sigma):
    ctr = m.geometry()["center"].reshape(3, -1).astype(np.float32)
    d = [ctr[k] - np.float32(c[k]) for k in range(3)]
    return np.exp(-(d[0] ** 2 + d[1] ** 2 + d[2] ** 2) / (2 * sigma * sigma)).astype(np.float64)


def test_heat_template_runs_fused_and_matches_oracle(oracle, tmp_path):
    n, steps = 16, 30
    (T,), out = run_example(tmp_path, "heat", n, n, n, steps)
    assert "fused_equations=1" in out
    m = oracle.Mesh(n, n, n, 1 / n, 1 / n, 1 / n)
    T0 = gaussian(m, (0.5, 0.5, 0.5), 0.1)
    dt = float(np.float32(0.1 * (1 / n) ** 2 / 0.01))
    ref = m.heat_solve(T0, 0.01, dt, steps)
    assert rel_l2(T, ref) <= 1e-5


def test_heat_with_device_boundary_copy(oracle, tmp_path):
    n, steps = 12, 20
    (T,), out = run_example(tmp_path, "heat_bc", n, n, n, steps)
    m = oracle.Mesh(n, n, n, 1 / n, 1 / n, 1 / n)
    T0 = gaussian(m, (0.5, 0.5, 0.5), 0.1)
    isb = m.geometry()["is_boundary"] > 0
    dt = float(np.float32(0.1 * (1 / n) ** 2 / 0.01))
    ref = T0.copy()
    for _ in range(steps):
        ref = m.heat_solve(ref, 0.01, dt, 1)
        ref[isb] = T0[isb]  # _boundary_copy_cu after every step
    assert rel_l2(T, ref) <= 1e-5


def test_d2t_leapfrog_operator_tree(oracle, tmp_path):
    """d2t(u) = c^2 (d2dx(u) + d2dy(u)) -- the scheme of examples/main_3d_wave.cu."""
    n, steps = 16, 25
    (U,), _ = run_example(tmp_path, "wave_d2t", n, n, n, steps)
    m = oracle.Mesh(n, n, n, 1 / n, 1 / n, 1 / n)
    u = gaussian(m, (0.5, 0.5, 0.5), 0.15)
    prev = None
    dt, c = 0.01, 0.3
    for _ in range(steps):
        R = c * c * (m.lapl(u, 1) + m.lapl(u, 2))
        nxt = dt * R + u if prev is None else (dt * dt * R + 2 * u) - prev
        prev, u = u, nxt
    assert rel_l2(U, u) <= 1e-5


@pytest.mark.parametrize("mode,nfields,n", [("advect", 2, 12), ("wave_d2t", 1, 16), ("advect", 2, 9),
                                            ("advect", 2, 16), ("wave_d2t", 1, 13), ("nested", 1, 16),
                                            ("nested", 1, 11)])
def test_jit_equations_equal_operator_path_bitwise(tmp_path, mode, nfields, n):
    """use_jit equations run as generated kernels (KernelBuilder,
    src/fvm3d.cpp:1219-1394): grad, lapl and the two-stage stab of
    expressions, a plain left-hand side, d1t and d2t.  The generated kernel
    rounds like the operator-by-operator path (--fmad=false, same operand
    order), so both give the same bits.  dx = 1/16 is an exact lattice: the
    kernels take the geometry as constants, and the face-array form
    (_arrays) gives the same bits too; n = 9, 11, 13 have nz % 4 != 0.
    nested: operands holding operators, materialised in passes of their own.
    advect: the second equation reads q at neighbours after the first wrote
    it, so the two run as two kernels."""
    steps = 7
    (J, out_j) = run_example(tmp_path, mode, n, n, n, steps, nfields)
    (P, out_p) = run_example(tmp_path, mode + "_nojit", n, n, n, steps, nfields)
    (A, out_a) = run_example(tmp_path, mode + "_arrays", n, n, n, steps, nfields)
    jit_eqs = 2 if mode == "advect" else 1
    assert "jit_equations=0" in out_p and "fused_equations=0" in out_p
    if mode == "wave_d2t" and n % 4 == 0:
        # the wave template on an exact lattice runs as one fused pass (cfdb_d2t_step)
        assert "fused_equations=1" in out_j and "jit_equations=0" in out_j
        assert "jit_equations=1" in out_a and "fused_equations=0" in out_a
    else:
        assert f"jit_equations={jit_eqs}" in out_j
        if n == 16:
            assert f"lattice_equations={jit_eqs}" in out_j
    if mode == "advect":
        assert "jit_groups=2" in out_j
    assert "lattice_equations=0" in out_a
    assert np.array_equal(J, P)
    assert np.array_equal(A, P)


@pytest.mark.parametrize("n", [16, 13])
def test_reference_euler_system_jit_equals_operator_path(tmp_path, n):
    """The reference's 3-D Euler benchmark system (examples/main_3d.cpp: 15
    use_jit equations incl. d1dx of products, 5 use_jit = false updates with
    stab_tot of products, CFL time step, Dirichlet boundary layers) on unit
    cells, an exact lattice.  All 20 run as generated kernels (geometry as
    constants, and as face arrays) and give the bits of the operator path,
    hence of any split between the two; the state stays finite."""
    steps = 6
    J, out_j = run_example(tmp_path, "euler3d", n, n, n, steps, 5)
    P, out_p = run_example(tmp_path, "euler3d_nojit", n, n, n, steps, 5)
    A, out_a = run_example(tmp_path, "euler3d_arrays", n, n, n, steps, 5)
    assert "jit_equations=20" in out_j and "jit_equations=0" in out_p
    assert "lattice_equations=20" in out_j and "lattice_equations=0" in out_a
    # fused into 4 kernels: [rho, u, v, w, p recovery], [predictor rho, u, v, w],
    # [predictor p, mass flux], [4 fluxes + 5 updates]
    assert "jit_groups=4" in out_j
    assert np.isfinite(J).all()
    assert np.array_equal(J, P)
    assert np.array_equal(A, P)


@pytest.mark.parametrize("n,steps", [(16, 20), (13, 12)])
def test_reference_euler_system_matches_oracle(oracle, tmp_path, n, steps):
    """The reference's 20-equation Euler system (examples/main_3d.cpp:238-263)
    as the example runs it on the GPU (generated kernels, FP32) against the
    oracle's run of the same system (oracle/euler_system.py: the CPU path's
    loop order of src/fvm3d.cpp:1008-1049 over the restated operators),
    started from the example's own initial state (a 0-step run).  Against
    the FP64 run every field is within 1e-5 (rel L2); against the FP32 run,
    which rounds like the reference, within 1e-6."""
    from oracle import euler_system as ES
    init, _ = run_example(tmp_path, "euler3d", n, n, n, 0, 5)
    J, out = run_example(tmp_path, "euler3d", n, n, n, steps, 5)
    assert "jit_equations=20" in out
    prim0 = [init[k].astype(np.float32) for k in range(5)]
    ref64, dts = ES.run(n, n, n, steps, *prim0, dtype=np.float64)
    ref32, _ = ES.run(n, n, n, steps, *prim0, dtype=np.float32)
    moved = max(rel_l2(ref64[k], init[k]) for k in range(5))
    assert moved > 1e-4  # the state has evolved
    for k, name in enumerate(("rho", "u", "v", "w", "p")):
        e64, e32 = rel_l2(J[k], ref64[k]), rel_l2(J[k], ref32[k])
        print(f"{name}: rel L2 vs FP64 oracle {e64:.2e}, vs FP32 oracle {e32:.2e}, "
              f"bitwise FP32 {np.array_equal(J[k], ref32[k].astype(np.float64))}")
        assert e64 <= 1e-5, (name, e64)
        assert e32 <= 1e-6, (name, e32)


def test_jit_heat_on_a_mesh_the_sweep_cannot_take(oracle, tmp_path):
    """The heat template on nz % 4 != 0 cannot use the fused TMA step; with
    use_jit it runs as a generated kernel and matches the oracle."""
    n, steps = 10, 20
    (T,), out = run_example(tmp_path, "heat", n, n, n, steps)
    assert "fused_equations=0" in out and "jit_equations=1" in out
    m = oracle.Mesh(n, n, n, 1 / n, 1 / n, 1 / n)
    T0 = gaussian(m, (0.5, 0.5, 0.5), 0.1)
    dt = float(np.float32(0.1 * (1 / n) ** 2 / 0.01))
    assert rel_l2(T, m.heat_solve(T0, 0.01, dt, steps)) <= 1e-5


def test_reference_heat_benchmark_row(oracle, tmp_path):
    """examples/main_3d_heat.cpp as its benchmark runs it: unit cells, T = 100
    in the two lowest z layers, d1t(T) = 3 lapl(T), dt 0.005, the boundary
    cells copied back from T0 after every step (fused step + device copy)."""
    n, steps = 12, 25
    (T,), out = run_example(tmp_path, "ref_heat", n, n, n, steps)
    assert "fused_equations=1" in out and "evaluate_us=" in out
    m = oracle.Mesh(n, n, n, 1.0, 1.0, 1.0)
    z = m.geometry()["center"].reshape(3, -1)[2].astype(np.float32)
    T0 = np.where(z < 2.0, 100.0, 0.0)
    isb = m.geometry()["is_boundary"] > 0
    ref = T0.copy()
    for _ in range(steps):
        ref = m.heat_solve(ref, 3.0, float(np.float32(0.005)), 1)
        ref[isb] = T0[isb]
    assert rel_l2(T, ref) <= 1e-5


def test_reference_wave_benchmark_row(oracle, tmp_path):
    """examples/main_3d_wave.cu as its benchmark runs it: u = 0, d2t(u) =
    c^2 (d2dx(u) + d2dy(u)) with c 0.3 and dt 0.1, and after every step the
    cells at 0.1 and 0.9 of the box set to sin(0.2 step) (step counted from
    1, computed in double and stored as float)."""
    n, steps = 10, 30
    (U,), out = run_example(tmp_path, "ref_wave", n, n, n, steps)
    assert "jit_equations=1" in out
    m = oracle.Mesh(n, n, n, 1.0, 1.0, 1.0)
    n1 = n * n * int(n * 0.1) + n * int(n * 0.1) + int(n * 0.1)
    n2 = n * n * int(n * 0.9) + n * int(n * 0.9) + int(n * 0.9)
    u = np.zeros(n ** 3)
    prev = None
    dt, c = float(np.float32(0.1)), float(np.float32(0.3))
    for t in range(1, steps + 1):
        R = c * c * (m.lapl(u, 1) + m.lapl(u, 2))
        nxt = dt * R + u if prev is None else (dt * dt * R + 2 * u) - prev
        prev, u = u, nxt
        u[[n1, n2]] = float(np.float32(np.sin(float(np.float32(t)) * 0.2)))
    assert np.abs(U).max() > 0.1
    assert rel_l2(U, u) <= 1e-5


def test_store_history_files(oracle, tmp_path):
    """The reference's output calls through the facade: store_history writes
    <store_dir>/T/res_<i>.vti for every stored step but the last and links
    run_latest; the stepping calls write mesh.json and a raw .bin of the
    final state."""
    import json
    from test_io_cpu import read_vti
    n, steps = 8, 5
    store = tmp_path / "dumps"
    out = tmp_path / "heat_store.bin"
    r = subprocess.run([EXE, "heat_store", str(out), str(n), str(n), str(n), str(steps), str(store)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    runs = [p for p in store.iterdir() if p.name.startswith("run_") and p.name != "run_latest"]
    assert len(runs) == 1
    run = runs[0]
    assert (store / "run_latest").resolve() == run.resolve()
    m = oracle.Mesh(n, n, n, 1 / n, 1 / n, 1 / n)
    T = gaussian(m, (0.5, 0.5, 0.5), 0.1)
    dt = float(np.float32(0.1 * (1 / n) ** 2 / 0.01))
    vtis = sorted((run / "T").glob("res_*.vti"), key=lambda p: int(p.stem[4:]))
    assert [p.name for p in vtis] == [f"res_{i}.vti" for i in range(steps - 1)]
    x, y, z = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    for i, p in enumerate(vtis):
        T = m.heat_solve(T, 0.01, dt, 1)
        _, img = read_vti(p)
        cells = np.empty(n ** 3, np.float32)
        cells[n * n * x + n * y + z] = img[x + n * (y + n * z)]
        assert rel_l2(cells.astype(np.float64), T) <= 1e-5, i
    mesh = json.loads((run / "mesh.json").read_text())
    assert len(mesh["nodes"]) == n ** 3 and mesh["x"] == n
    final = np.fromfile(run / "T" / f"{steps}.bin", dtype=np.float32)
    assert np.array_equal(final, np.fromfile(out, dtype=np.float32))


def test_operator_tree_with_grad_stab_and_sequential_equations(oracle, tmp_path):
    n, steps = 12, 15
    (Q, R), _ = run_example(tmp_path, "advect", n, n, n, steps, nfields=2)
    m = oracle.Mesh(n, n, n, 1 / n, 1 / n, 1 / n)
    q = gaussian(m, (0.4, 0.5, 0.5), 0.15)
    r = np.zeros_like(q)
    u, v, dt = 0.3, -0.2, float(np.float32(0.002))
    for _ in range(steps):
        q = q - dt * (u * m.grad(q, 1) + v * m.grad(q, 2)) + 0.01 * m.stab(q)
        r = dt * (-m.grad(q, 4) - r) + r  # sees the q updated by the first equation
    # FP32 operator tree (upwind extrapolation + opposite-face jumps in stab
    # cancel to ~1e-6 of the field) against FP64: 1e-4 relative L2
    assert rel_l2(Q, q) <= 1e-4
    assert rel_l2(R, r) <= 1e-4


def test_generated_kernels_report_no_spills(tmp_path):
    """_report prints each generated kernel's resources (cfdb_kernel_info):
    the reference's Euler system builds its fused groups (4, plus any
    materialised operand passes), none spilling to local memory, and the
    report changes no result."""
    n, steps = 16, 4
    out = tmp_path / "report.bin"
    r = subprocess.run([EXE, "euler3d_report", str(out), str(n), str(n), str(n), str(steps)], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stderr.splitlines() if ln.startswith("jit kernel ")]
    assert len(lines) >= 4, r.stderr
    for ln in lines:
        regs = int(ln.split(", ")[1].split()[0])
        local = int(ln.split(", ")[2].split()[0])
        assert 0 < regs <= 255 and local == 0, ln
    plain, _ = run_example(tmp_path, "euler3d", n, n, n, steps, 5)
    assert np.array_equal(np.fromfile(out, dtype=np.float32).astype(np.float64).reshape(5, -1), plain)
