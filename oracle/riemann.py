"""TEST INFRASTRUCTURE ONLY: exact solution of the 1-D Riemann problem for
the ideal-gas Euler equations, after E. F. Toro, *Riemann Solvers and
Numerical Methods for Fluid Dynamics*, 3rd ed., ch. 4 (pressure function
with Newton iteration for p*, then sampling of the wave pattern).

It replaces the third-party ``sodshock`` package that the reference's Sod
validation script uses (reports/compare_sod_shock.py:52-65); that package is
not installed here.
"""
from __future__ import annotations

import math

import numpy as np


def _f_and_df(p, rho_k, p_k, a_k, g):
    if p > p_k:  # shock
        A = 2.0 / ((g + 1.0) * rho_k)
        B = (g - 1.0) / (g + 1.0) * p_k
        s = math.sqrt(A / (p + B))
        return (p - p_k) * s, s * (1.0 - 0.5 * (p - p_k) / (B + p))
    # rarefaction
    e = (g - 1.0) / (2.0 * g)
    f = 2.0 * a_k / (g - 1.0) * ((p / p_k) ** e - 1.0)
    df = 1.0 / (rho_k * a_k) * (p / p_k) ** (-(g + 1.0) / (2.0 * g))
    return f, df


def star_state(rl, ul, pl, rr, ur, pr, g=1.4, tol=1e-14):
    al, ar = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    # two-rarefaction initial guess (Toro eq. 4.46)
    e = (g - 1.0) / (2.0 * g)
    p = ((al + ar - 0.5 * (g - 1.0) * (ur - ul)) / (al / pl ** e + ar / pr ** e)) ** (1.0 / e)
    p = max(p, tol)
    for _ in range(200):
        fl, dfl = _f_and_df(p, rl, pl, al, g)
        fr, dfr = _f_and_df(p, rr, pr, ar, g)
        dp = (fl + fr + (ur - ul)) / (dfl + dfr)
        pn = max(p - dp, tol)
        if abs(pn - p) <= tol * 0.5 * (pn + p):
            p = pn
            break
        p = pn
    fl, _ = _f_and_df(p, rl, pl, al, g)
    fr, _ = _f_and_df(p, rr, pr, ar, g)
    u = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    return p, u


def sample(x, t, x0, left, right, g=1.4):
    """Density, velocity, pressure at positions x and time t > 0."""
    rl, ul, pl = left
    rr, ur, pr = right
    ps, us = star_state(rl, ul, pl, rr, ur, pr, g)
    al, ar = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    out = np.zeros((3, len(x)))
    for k, xi in enumerate(np.asarray(x, dtype=np.float64)):
        s = (xi - x0) / t
        if s <= us:  # left of contact
            if ps > pl:  # left shock
                sl = ul - al * math.sqrt((g + 1) / (2 * g) * ps / pl + (g - 1) / (2 * g))
                if s <= sl:
                    r, u, p = rl, ul, pl
                else:
                    r = rl * ((ps / pl + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pl + 1))
                    u, p = us, ps
            else:  # left rarefaction
                shl = ul - al
                asl = al * (ps / pl) ** ((g - 1) / (2 * g))
                stl = us - asl
                if s <= shl:
                    r, u, p = rl, ul, pl
                elif s > stl:
                    r, u, p = rl * (ps / pl) ** (1 / g), us, ps
                else:
                    c = 2 / (g + 1) + (g - 1) / ((g + 1) * al) * (ul - s)
                    r = rl * c ** (2 / (g - 1))
                    u = 2 / (g + 1) * (al + (g - 1) / 2 * ul + s)
                    p = pl * c ** (2 * g / (g - 1))
        else:  # right of contact
            if ps > pr:  # right shock
                sr = ur + ar * math.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
                if s >= sr:
                    r, u, p = rr, ur, pr
                else:
                    r = rr * ((ps / pr + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pr + 1))
                    u, p = us, ps
            else:  # right rarefaction
                shr = ur + ar
                asr = ar * (ps / pr) ** ((g - 1) / (2 * g))
                str_ = us + asr
                if s >= shr:
                    r, u, p = rr, ur, pr
                elif s <= str_:
                    r, u, p = rr * (ps / pr) ** (1 / g), us, ps
                else:
                    c = 2 / (g + 1) - (g - 1) / ((g + 1) * ar) * (ur - s)
                    r = rr * c ** (2 / (g - 1))
                    u = 2 / (g + 1) * (-ar + (g - 1) / 2 * ur + s)
                    p = pr * c ** (2 * g / (g - 1))
        out[:, k] = (r, u, p)
    return out
