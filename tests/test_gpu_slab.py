"""The fused GPU steps under the x-slab split (cfdarcov2_b200/slab.py): two
slabs of one mesh advanced in one process, their ghost planes copied between
them on the device before every step (what the exchange does between
ranks), give the undivided fused run's bits.  This holds because the sweep
kernels read only spacings and neighbour values, never absolute positions."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.mark.parametrize("case", ["wave", "heat"])
def test_two_slabs_equal_the_undivided_fused_run(cfdb, ctx, case):
    from cfdarcov2_b200.slab import split
    nx, ny, nz, steps = 37, 24, 32, 11
    nf = 4 if case == "wave" else 1
    h = 1.0 / 32
    rng = np.random.default_rng(5)
    q0 = torch.tensor(rng.standard_normal(nf * nx * ny * nz), dtype=torch.float32, device=DEV)
    plane = ny * nz

    def step(mesh, a, b):
        if case == "wave":
            ctx.wave_step(mesh, a, b, 0.4 * h / 3, path=cfdb.FUSED)
        else:
            ctx.heat_step(mesh, a, b, 0.01, 0.1 * h * h / 0.01, path=cfdb.FUSED)

    full_mesh = cfdb.Mesh.structured(ctx, nx, ny, nz, h, h, h)
    a, b = q0.clone(), torch.empty_like(q0)
    for _ in range(steps):
        step(full_mesh, a, b)
        a, b = b, a
    ref = a.clone()

    # two slabs: planes [0, x1) + 1 ghost, and 1 ghost + [x1, nx)
    x1 = split(nx, 2, 0)[1]
    parts = []
    for lo, hi in ((0, x1 + 1), (x1 - 1, nx)):
        lnx = hi - lo
        m = cfdb.Mesh.structured(ctx, lnx, ny, nz, h, h, h)
        la = torch.cat([q0[f * nx * plane + lo * plane: f * nx * plane + hi * plane] for f in range(nf)])
        parts.append([m, lnx, la, torch.empty_like(la)])

    def pl(p, f, i):
        lnx = p[1]
        o = (f * lnx + i) * plane
        return p[2][o: o + plane]

    for _ in range(steps):
        for f in range(nf):  # the exchange: last owned plane of slab 0 <-> first owned plane of slab 1
            pl(parts[0], f, parts[0][1] - 1).copy_(pl(parts[1], f, 1))
            pl(parts[1], f, 0).copy_(pl(parts[0], f, parts[0][1] - 2))
        for p in parts:
            step(p[0], p[2], p[3])
            p[2], p[3] = p[3], p[2]
    got = torch.empty_like(ref)
    for f in range(nf):
        got[f * nx * plane: f * nx * plane + x1 * plane] = parts[0][2][f * parts[0][1] * plane:
                                                                      (f * parts[0][1] + x1) * plane]
        o = (f * parts[1][1] + 1) * plane
        got[f * nx * plane + x1 * plane: (f + 1) * nx * plane] = parts[1][2][o: o + (nx - x1) * plane]
    assert torch.equal(got, ref)
