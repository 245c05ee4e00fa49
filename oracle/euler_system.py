"""TEST INFRASTRUCTURE ONLY: the reference's 20-equation Euler benchmark system
run on the CPU restatement's operators.

Restates examples/main_3d.cpp:187-263 (variables, initial conservative
values, the equation list) under the time loop of Equation::evaluate
(src/fvm3d.cpp:1008-1049):

  * DT::update first (src/fvm3d.cpp:641-662) with the CourantFriedrichsLewy3D
    policy (src/fvm3d.cpp:512-528): dt = CFL * dl / max_P(sqrt(gamma p / rho)
    + |u|), gamma = 5/3, dl = min(dx, dy, dz); the reference keeps dt as a
    float;
  * the equations in list order, each one's right-hand side evaluated over
    the whole mesh from the current values (the earlier equations of the same
    step already applied) and then stored: a plain left-hand side takes the
    value (the CPU path's Variable::solve), d1t(x) takes x + dt * rhs
    (DtVar::extract, src/fvm3d.cpp:690-692);
  * after the equations, the boundary cells of the ten state variables are
    reset to their initial values (boundary_copy of the example; the _tmp
    variables and the volumes have no boundary function).

E is the example's expression variable p / (gamma - 1) + 0.5 rho (u^2 + v^2
+ w^2), evaluated from the current values where it is read.  d1dx/d1dy/d1dz
are the Green-Gauss gradient with dimension masks 1/2/4 (GradVar,
src/fvm3d.cpp:768-829) and stab_tot the two-stage stabilisation over all
dimensions (StabVar, src/fvm3d.cpp:909-942).

`dtype` selects the arithmetic: float32 repeats the reference's precision
operation by operation (Python evaluates the example's operator expressions
with C++'s left-to-right association), float64 gives the higher-precision
solution of the same discrete scheme.  Only tests may import this module.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O

GAMMA = 5.0 / 3.0  # the float constant of the example, `float gamma = 5. / 3.`
CFL = 0.005        # the example's default CFL (include/utils3d.hpp:35-66)
DISSIP = 2.0


def run(nx, ny, nz, steps, rho0, u0, v0, w0, p0, dtype=np.float64, dx=1.0, dy=1.0, dz=1.0):
    """Runs `steps` time steps of the system on an nx x ny x nz mesh (unit
    cells by default, as the reference's benchmark) from the float32 initial
    primitives (rho0, u0, v0, w0, p0; cell order z fastest).  Returns the
    final (rho, u, v, w, p) and the dt of every step."""
    R = np.dtype(dtype).type
    f32 = np.float32
    m = O.Mesh(nx, ny, nz, dx, dy, dz, dtype=dtype)
    geo = m.geometry()
    bnd = geo["is_boundary"] > 0
    n = m.n

    # initial conservative values, computed in float as the example does
    prim = [np.asarray(a, f32) for a in (rho0, u0, v0, w0, p0)]
    r, u, v, w, p = prim
    g32 = f32(GAMMA)
    vol32 = np.full(n, f32(dx) * f32(dy) * f32(dz), f32)
    mass0 = r * vol32
    rho_u0 = r * u * vol32
    rho_v0 = r * v * vol32
    rho_w0 = r * w * vol32
    rho_e0 = (p / (g32 - f32(1)) + f32(0.5) * r * (u * u + v * v + w * w)) * vol32

    def cast(a):
        return np.asarray(a, dtype).copy()

    state = {k: cast(a) for k, a in (("rho", r), ("u", u), ("v", v), ("w", w), ("p", p), ("mass", mass0),
                                      ("rho_u", rho_u0), ("rho_v", rho_v0), ("rho_w", rho_w0),
                                      ("rho_e", rho_e0))}
    init = {k: a.copy() for k, a in state.items()}
    tmp = {k: cast(a) for k, a in (("mass_tmp", mass0), ("rho_u_tmp", rho_u0), ("rho_v_tmp", rho_v0),
                                    ("rho_w_tmp", rho_w0), ("rho_e_tmp", rho_e0))}
    vol = cast(vol32)
    gamma = R(g32)
    half = R(0.5)
    one = R(1)
    zero = R(0)
    dissip = R(DISSIP)

    def gx(a):
        return m.grad(a, 1)

    def gy(a):
        return m.grad(a, 2)

    def gz(a):
        return m.grad(a, 4)

    def stab(a):
        return m.stab(a, 7)

    dts = []
    for _ in range(steps):
        S = state
        dt_val = m.cfl_reference(CFL, GAMMA, S["p"], S["rho"], S["u"], S["v"], S["w"])
        dt = R(f32(dt_val)) if R is np.float32 else R(dt_val)
        dts.append(float(dt))

        S["rho"] = S["mass"] / vol
        S["u"] = S["rho_u"] / S["rho"] / vol
        S["v"] = S["rho_v"] / S["rho"] / vol
        S["w"] = S["rho_w"] / S["rho"] / vol
        rho, u, v, w = S["rho"], S["u"], S["v"], S["w"]
        S["p"] = (S["rho_e"] / vol - half * rho * (u * u + v * v + w * w)) * (gamma - one)
        p = S["p"]

        hdt = half * dt
        S["rho"] = rho - hdt * (u * gx(rho) + rho * gx(u) + v * gy(rho) + rho * gy(v) + w * gz(rho) + rho * gz(w))
        rho = S["rho"]
        S["u"] = u - hdt * (u * gx(u) + v * gy(u) + w * gz(u) + (one / rho) * gx(p))
        u = S["u"]
        S["v"] = v - hdt * (u * gx(v) + v * gy(v) + w * gz(v) + (one / rho) * gy(p))
        v = S["v"]
        S["w"] = w - hdt * (u * gx(w) + v * gy(w) + w * gz(w) + (one / rho) * gz(p))
        w = S["w"]
        S["p"] = p - hdt * (gamma * p * (gx(u) + gy(v) + gz(w)) + u * gx(p) + v * gy(p) + w * gz(p))
        p = S["p"]

        T = tmp
        T["mass_tmp"] = zero * T["mass_tmp"] - (gx(rho * u) + gy(rho * v) + gz(rho * w))
        T["rho_u_tmp"] = zero * T["rho_u_tmp"] - (gx(rho * u * u + p) + gy(rho * v * u) + gz(rho * w * u))
        T["rho_v_tmp"] = zero * T["rho_v_tmp"] - (gx(rho * v * u) + gy(rho * v * v + p) + gz(rho * v * w))
        T["rho_w_tmp"] = zero * T["rho_w_tmp"] - (gx(rho * w * u) + gy(rho * w * v) + gz(rho * w * w + p))
        E = p / (gamma - one) + half * rho * ((u * u) + (v * v) + (w * w))
        T["rho_e_tmp"] = zero * T["rho_e_tmp"] - (gx((E + p) * u) + gy((E + p) * v) + gz((E + p) * w))

        S["mass"] = dt * (T["mass_tmp"] - stab(rho) * dissip) + S["mass"]
        S["rho_u"] = dt * (T["rho_u_tmp"] - stab(rho * u) * dissip) + S["rho_u"]
        S["rho_v"] = dt * (T["rho_v_tmp"] - stab(rho * v) * dissip) + S["rho_v"]
        S["rho_w"] = dt * (T["rho_w_tmp"] - stab(rho * w) * dissip) + S["rho_w"]
        E = p / (gamma - one) + half * rho * ((u * u) + (v * v) + (w * w))
        S["rho_e"] = dt * (T["rho_e_tmp"] - stab(E) * dissip) + S["rho_e"]

        for k in S:  # boundary_copy of every state variable
            S[k][bnd] = init[k][bnd]
    return tuple(state[k] for k in ("rho", "u", "v", "w", "p")), dts
