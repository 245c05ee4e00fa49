"""Seeded synthetic inputs for the five benchmark workloads.

All randomness comes from numpy PCG64 generators with the seeds stated per
workload, so the GPU path and the CPU oracle see identical inputs.
  heat      64^3 on [0,1]^3, k = 0.01, dt = 0.1 dx^2 / k, 200 steps (seed 1)
  wave      128^3 on [0,1]^3, c = 1, Gaussian pulse sigma 0.05, CFL 0.4, 500 steps
  wave_dist the same on vertices jittered by U(-0.2, 0.2) dx (seed 2)
  sod       512 x 64 x 64 on [0,1] x [0,0.125]^2, gamma 1.4, CFL 0.4, t = 0.2
  ensemble  512 cubes, n log-uniform in [16, 96] (seed 4), heat or wave
  adjoint   128^3, 400 steps, c = exp(0.2 g), g a Gaussian random field (seed 5)
"""
from __future__ import annotations

import math

import numpy as np


def cell_centers(nx, ny, nz, dx, dy, dz):
    """Cell centres in reference order (id = Z*Y*x + Z*y + z), shape (3, n)."""
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dy
    z = (np.arange(nz) + 0.5) * dz
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    return np.stack([X.reshape(-1), Y.reshape(-1), Z.reshape(-1)])


# ---- heat ---------------------------------------------------------------------
def heat_config(n=64, k=0.01, steps=200, seed=1):
    dx = 1.0 / n
    dt = 0.1 * dx * dx / k
    c = cell_centers(n, n, n, dx, dx, dx)
    r2 = ((c - 0.5) ** 2).sum(axis=0)
    rng = np.random.Generator(np.random.PCG64(seed))
    T0 = np.exp(-r2 / (2 * 0.1 ** 2)) + rng.uniform(-1e-3, 1e-3, size=r2.shape)
    return dict(n=n, dx=dx, k=k, dt=dt, steps=steps, T0=T0)


# ---- wave ---------------------------------------------------------------------
def wave_state(n, sigma=0.05, center=(0.5, 0.5, 0.5)):
    dx = 1.0 / n
    c = cell_centers(n, n, n, dx, dx, dx)
    r2 = sum((c[d] - center[d]) ** 2 for d in range(3))
    q = np.zeros(4 * n ** 3)
    q[: n ** 3] = np.exp(-r2 / (2 * sigma ** 2))
    return q


def wave_config(n=128, c=1.0, cfl=0.4, steps=500):
    dx = 1.0 / n
    dt = cfl / (3 * c / dx)
    return dict(n=n, dx=dx, c=c, cfl=cfl, dt=dt, steps=steps, q0=wave_state(n))


def jittered_vertices(n, amp=0.2, seed=2):
    """(n+1)^3 x 3 lattice on [0,1]^3 jittered by U(-amp, amp) dx per coordinate;
    a vertex on a wall keeps its wall-normal coordinate so the domain stays the
    unit cube."""
    dx = 1.0 / n
    rng = np.random.Generator(np.random.PCG64(seed))
    g = np.arange(n + 1) * dx
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    V = np.stack([X, Y, Z], axis=-1)
    J = rng.uniform(-amp, amp, size=V.shape) * dx
    idx = np.arange(n + 1)
    on_wall = (idx == 0) | (idx == n)
    J[on_wall, :, :, 0] = 0.0
    J[:, on_wall, :, 1] = 0.0
    J[:, :, on_wall, 2] = 0.0
    return (V + J).reshape(-1, 3)


# ---- Sod ----------------------------------------------------------------------
def sod_state(nx=512, ny=64, nz=64, lx=1.0, lyz=0.125, gamma=1.4):
    dx, dy, dz = lx / nx, lyz / ny, lyz / nz
    xc = (np.arange(nx) + 0.5) * dx
    left = xc < 0.5 * lx
    rho1 = np.where(left, 1.0, 0.125)
    p1 = np.where(left, 1.0, 0.1)
    n = nx * ny * nz
    rho = np.repeat(rho1, ny * nz)
    p = np.repeat(p1, ny * nz)
    U = np.zeros(5 * n)
    U[:n] = rho
    U[4 * n:] = p / (gamma - 1.0)
    return U, (dx, dy, dz)


def sod_config(nx=512, ny=64, nz=64):
    U0, (dx, dy, dz) = sod_state(nx, ny, nz)
    return dict(nx=nx, ny=ny, nz=nz, dx=dx, dy=dy, dz=dz, gamma=1.4, cfl=0.4, t_end=0.2, U0=U0)


# ---- ensemble -------------------------------------------------------------------
def ensemble_problems(count=512, nmin=16, nmax=96, seed=4, kinds="mixed"):
    """Problem list: n log-uniform in [nmin, nmax]; even index heat
    (k ~ U(1e-3, 1e-2), dt = 0.1 dx^2/k), odd index wave (c ~ U(0.5, 2),
    dt = 0.4 dx / (3 c)), unless kinds is "heat" or "wave"."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ns = np.floor(np.exp(rng.uniform(math.log(nmin), math.log(nmax + 1), size=count))).astype(int)
    ns = np.clip(ns, nmin, nmax)
    ks = rng.uniform(1e-3, 1e-2, size=count)
    cs = rng.uniform(0.5, 2.0, size=count)
    centers = rng.uniform(0.3, 0.7, size=(count, 3))
    probs = []
    for i in range(count):
        kind = {"heat": 0, "wave": 1}.get(kinds, i % 2)
        n = int(ns[i])
        dx = 1.0 / n
        if kind == 0:
            probs.append(dict(n=n, kind=0, param=float(ks[i]), dt=0.1 * dx * dx / float(ks[i]), center=centers[i]))
        else:
            probs.append(dict(n=n, kind=1, param=float(cs[i]), dt=0.4 * dx / (3 * float(cs[i])), center=centers[i]))
    return probs


def ensemble_initial(probs, offsets, pool_elems, sigma=0.1):
    pool = np.zeros(pool_elems, np.float32)
    for p, off in zip(probs, offsets):
        n = p["n"]
        dx = 1.0 / n
        c = cell_centers(n, n, n, dx, dx, dx)
        r2 = sum((c[d] - p["center"][d]) ** 2 for d in range(3))
        pool[off: off + n ** 3] = np.exp(-r2 / (2 * sigma ** 2))
    return pool


# ---- adjoint --------------------------------------------------------------------
def gaussian_random_field(n, corr=0.1, seed=5):
    """Unit-variance periodic Gaussian random field on the n^3 cell grid: white
    noise filtered in Fourier space by a Gaussian kernel of correlation
    length corr (in domain units)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = rng.standard_normal((n, n, n))
    k = np.fft.fftfreq(n, d=1.0 / n) * 2 * np.pi
    KX, KY, KZ = np.meshgrid(k, k, k, indexing="ij")
    filt = np.exp(-0.5 * (KX ** 2 + KY ** 2 + KZ ** 2) * corr ** 2)
    g = np.real(np.fft.ifftn(np.fft.fftn(w) * filt))
    g = (g - g.mean()) / g.std()
    return g.reshape(-1)


def adjoint_config(n=128, steps=400, cfl=0.4):
    g = gaussian_random_field(n, seed=5)
    c = np.exp(0.2 * g)
    g2 = gaussian_random_field(n, seed=6)
    c_true = np.exp(0.2 * g2)
    dx = 1.0 / n
    dt = cfl / (3 * max(c.max(), c_true.max()) / dx)
    q0 = wave_state(n)
    return dict(n=n, dx=dx, steps=steps, dt=dt, c=c, c_true=c_true, q0=q0)
