"""Generates tests/golden/oracle_golden.npz: small seeded inputs and the CPU
oracle's outputs for them (geometry, every operator, a few time steps of each
scheme).  The reference cannot be run here, so these fixtures pin the oracle
against regressions rather than against reference output; the GPU parity
tests compare the C ABI against the same cases.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def compute_cases(O):
    from cfdarcov2_b200.workloads import jittered_vertices, sod_state, wave_state
    out = {}
    rng = np.random.Generator(np.random.PCG64(2024))
    # uniform mesh 5 x 6 x 7, anisotropic spacing
    m = O.Mesh(5, 6, 7, 0.2, 1 / 6, 1 / 7)
    phi = rng.standard_normal(m.n)
    out["u_phi"] = phi
    out["u_grad"] = m.grad(phi, 7)
    out["u_grad_x"] = m.grad(phi, 1)
    out["u_lapl"] = m.lapl(phi, 7)
    out["u_lapl_yz"] = m.lapl(phi, 6)
    out["u_stab"] = m.stab(phi, 7)
    out["u_stab_x"] = m.stab(phi, 1)
    out["u_heat10"] = m.heat_solve(phi, 0.02, 0.001, 10)
    q = rng.standard_normal(4 * m.n)
    out["u_q"] = q
    out["u_wave5"] = m.wave_solve(q, m.wave_dt(0.4), 5)
    # jittered mesh 6^3
    V = jittered_vertices(6, seed=2)
    md = O.Mesh(6, 6, 6, 1 / 6, 1 / 6, 1 / 6, vertices=V)
    g = md.geometry()
    for k in ("normal", "normal_alt", "area", "alpha_d", "len_c2f", "volume"):
        out["d_" + k] = g[k]
    phid = rng.standard_normal(md.n)
    out["d_phi"] = phid
    out["d_grad"] = md.grad(phid)
    out["d_lapl"] = md.lapl(phid)
    out["d_stab"] = md.stab(phid)
    qd = wave_state(6, sigma=0.2)
    out["d_wave10"] = md.wave_solve(qd, md.wave_dt(0.4), 10)
    # Sod 32 x 4 x 4, 20 steps worth of time
    U0, (dx, dy, dz) = sod_state(32, 4, 4, 1.0, 0.125)
    ms = O.Mesh(32, 4, 4, dx, dy, dz)
    U, steps, t, tot = ms.euler_solve(U0, 1.4, 0.4, 0.02)
    out["s_U"] = U
    out["s_steps"] = np.array([steps])
    out["s_totals"] = tot
    return out


def main():
    from oracle import oracle as O
    O.build()
    cases = compute_cases(O)
    np.savez_compressed(os.path.join(HERE, "oracle_golden.npz"), **cases)
    print("wrote", len(cases), "arrays")


if __name__ == "__main__":
    main()
