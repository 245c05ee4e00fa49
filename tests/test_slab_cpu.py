"""x-slab decomposition (cfdarcov2_b200/slab.py) on two CPU ranks over gloo.

Each rank owns a balanced range of x planes plus ghost planes, exchanges
one plane per field per step with its neighbours, and advances its local
array with the single-mesh step; the owned cells then carry exactly the
undivided run's bits.  The step here is the CPU restatement (the GPU run
uses the library's kernels through the same driver).  The mesh is a
jittered vertex mesh, so each rank's geometry comes from the same absolute
vertex coordinates as the undivided mesh's.  Also: the dt minimum and FP64
sums across ranks (the reference's MPI_Allreduce, legacy/fvm.cpp:785)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, case, out_dir):
    import datetime

    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    import sys
    sys.path.insert(0, root)
    from cfdarcov2_b200.slab import Slab
    from cfdarcov2_b200.workloads import jittered_vertices, wave_state
    from oracle import oracle as O
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        nx, ny, nz, steps = 13, 6, 8, 9  # 13 planes: an uneven split
        V = jittered_vertices(max(nx, ny, nz), amp=0.15, seed=7)
        # a nx x ny x nz block of the jittered cube's vertices
        n1 = max(nx, ny, nz) + 1
        V = V.reshape(n1, n1, n1, 3)[: nx + 1, : ny + 1, : nz + 1].reshape(-1, 3).copy()
        h = 1.0 / (n1 - 1)
        nf = 4 if case == "wave" else 1
        rng = np.random.default_rng(3)
        q0 = rng.standard_normal(nf * nx * ny * nz)
        if case == "wave":
            q0[: nx * ny * nz] += wave_state(1)[0]
        slab = Slab(nx, ny, nz, nf)
        om = O.Mesh(slab.lnx, ny, nz, h, h, h, vertices=slab.local_vertices(V))
        dt = 0.02
        if case == "wave":
            def step(a, b):
                b.copy_(torch.from_numpy(om.wave_solve(a.numpy(), dt, 1)))
        else:
            def step(a, b):
                b.copy_(torch.from_numpy(om.heat_solve(a.numpy(), 0.05, dt, 1)))
        full = torch.tensor(q0, dtype=torch.float64)
        a = slab.scatter(full, torch.empty(slab.local_elems, dtype=torch.float64))
        b = torch.empty_like(a)
        fin = slab.run(a, b, steps, step)
        got = slab.gather(fin, torch.empty_like(full) if rank == 0 else None)
        # reductions: dt min over ranks, FP64 sums of the owned cells' totals
        dmin = slab.min_dt(0.5 + rank)
        own = [float(t.sum()) for t in slab.owned(fin)]
        tot = slab.sum_fp64(own)
        if rank == 0:
            gm = O.Mesh(nx, ny, nz, h, h, h, vertices=V)
            ref = gm.wave_solve(q0, dt, steps) if case == "wave" else gm.heat_solve(q0, 0.05, dt, steps)
            np.save(os.path.join(out_dir, f"{case}_got.npy"), got.numpy())
            np.save(os.path.join(out_dir, f"{case}_ref.npy"), ref)
            n3 = nx * ny * nz
            np.save(os.path.join(out_dir, f"{case}_tot.npy"),
                    np.array([tot, [float(ref[f * n3:(f + 1) * n3].sum()) for f in range(nf)]], dtype=np.float64))
            np.save(os.path.join(out_dir, f"{case}_dmin.npy"), np.array([dmin]))
            np.save(os.path.join(out_dir, f"{case}_split.npy"), np.array([slab.x0, slab.x1, slab.lnx]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", ["wave", "heat"])
def test_split_run_equals_undivided_run_bitwise(tmp_path, case):
    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(2, _free_port(), case, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(tmp_path / f"{case}_got.npy")
    ref = np.load(tmp_path / f"{case}_ref.npy")
    assert np.array_equal(got, ref)
    tot = np.load(tmp_path / f"{case}_tot.npy")
    assert np.allclose(tot[0], tot[1], rtol=1e-12, atol=1e-12)
    assert float(np.load(tmp_path / f"{case}_dmin.npy")[0]) == 0.5
    x0, x1, lnx = np.load(tmp_path / f"{case}_split.npy")
    assert (x0, x1, lnx) == (0, 6, 7)  # rank 0 of 13 planes: 6 owned + 1 ghost


def test_split_is_balanced_and_rejects_too_many_ranks():
    from cfdarcov2_b200.slab import split
    parts = [split(13, 4, r) for r in range(4)]
    assert parts[0][0] == 0 and parts[-1][1] == 13
    assert all(parts[i][1] == parts[i + 1][0] for i in range(3))
    assert max(b - a for a, b in parts) - min(b - a for a, b in parts) <= 1
    with pytest.raises(ValueError):
        split(3, 4, 0)
