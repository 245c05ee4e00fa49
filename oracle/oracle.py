"""TEST INFRASTRUCTURE ONLY: ctypes front end of the CPU restatement.

The oracle restates cfdARCO's finite-volume operators (reference files
src/mesh3d.cpp, include/grad_utils.hpp, include/custom_cuda_functions.hpp,
src/fvm3d.cpp) plus the Rusanov wave / Euler schemes and the discrete wave
adjoint that the B200 kernels implement.  Only tests/, the smoke check and
the CPU-baseline leg of bench.py may import it; the product never does.

Parity status: UNPINNED -- the reference cannot be built here (Eigen3, OCCA,
RMM are absent) and ships no golden vectors; see fv_oracle.hpp.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libfv_oracle.so")
_lib = None

_P = C.c_void_p
_I64 = C.c_int64
_D = C.c_double
_INT = C.c_int


def build(force: bool = False) -> str:
    """Compile the restatement with the Makefile beside this file."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        for suf in ("f64", "f32"):
            f = getattr(L, f"fvo_mesh_create_{suf}")
            f.restype = _P
            f.argtypes = [_I64, _I64, _I64, _D, _D, _D, _P, _INT]
            getattr(L, f"fvo_mesh_destroy_{suf}").argtypes = [_P]
            getattr(L, f"fvo_mesh_export_{suf}").argtypes = [_P] * 11
            for op in ("grad", "lapl", "stab"):
                getattr(L, f"fvo_{op}_{suf}").argtypes = [_P, _P, _P, _INT]
            f = getattr(L, f"fvo_cfl_reference_{suf}")
            f.restype = _D
            f.argtypes = [_P, _D, _D, _P, _P, _P, _P, _P]
            getattr(L, f"fvo_heat_solve_{suf}").argtypes = [_P, _P, _D, _D, _INT, _INT]
            f = getattr(L, f"fvo_heat_time_{suf}")
            f.restype = _D
            f.argtypes = [_P, _P, _D, _D, _INT, _INT]
            getattr(L, f"fvo_wave_rhs_{suf}").argtypes = [_P, _P, _P, _D, _INT, _P]
            getattr(L, f"fvo_wave_solve_{suf}").argtypes = [_P, _P, _P, _D, _INT, _D, _INT, _INT]
            f = getattr(L, f"fvo_wave_time_{suf}")
            f.restype = _D
            f.argtypes = [_P, _P, _D, _D, _INT, _INT]
            f = getattr(L, f"fvo_wave_dt_{suf}")
            f.restype = _D
            f.argtypes = [_P, _P, _D, _D]
            getattr(L, f"fvo_wave_adjoint_step_{suf}").argtypes = [_P, _P, _P, _P, _P, _P, _D]
            f = getattr(L, f"fvo_wave_gradient_{suf}")
            f.restype = _D
            f.argtypes = [_P, _P, _P, _P, _D, _INT, _P, _P]
            f = getattr(L, f"fvo_wave_objective_{suf}")
            f.restype = _D
            f.argtypes = [_P, _P, _P, _P, _D, _INT]
            getattr(L, f"fvo_euler_rhs_{suf}").argtypes = [_P, _P, _D, _P]
            f = getattr(L, f"fvo_euler_solve_{suf}")
            f.restype = _INT
            f.argtypes = [_P, _P, _D, _D, _D, _INT, _P, _P]
            f = getattr(L, f"fvo_total_{suf}")
            f.restype = _D
            f.argtypes = [_P, _P]
        L.fvo_max_threads.restype = _INT
        L.fvo_set_threads.argtypes = [_INT]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def set_threads(n: int) -> None:
    lib().fvo_set_threads(int(n))


def max_threads() -> int:
    return int(lib().fvo_max_threads())


class Mesh:
    """Mesh3D restated (src/mesh3d.cpp:151-385) in float64 or float32."""

    def __init__(self, nx, ny, nz, dx, dy, dz, vertices=None, dtype=np.float64, compat_area=False):
        self.dtype = np.dtype(dtype)
        self.suf = "f64" if self.dtype == np.float64 else "f32"
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.n = self.nx * self.ny * self.nz
        self.dx, self.dy, self.dz = float(dx), float(dy), float(dz)
        verts = None
        if vertices is not None:
            verts = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1)
            assert verts.size == 3 * (nx + 1) * (ny + 1) * (nz + 1)
        self._verts = verts
        # geometry mode: 0 reference formulas (uniform lattice), 1 reference with
        # the component-sum area, 2 exact vector areas (vertex meshes)
        mode = 1 if compat_area else (2 if verts is not None else 0)
        self.mode = mode
        self._h = getattr(lib(), f"fvo_mesh_create_{self.suf}")(
            self.nx, self.ny, self.nz, self.dx, self.dy, self.dz, _ptr(verts), mode)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                getattr(lib(), f"fvo_mesh_destroy_{self.suf}")(h)
            except TypeError:  # interpreter shutdown: module globals already cleared
                pass
            self._h = None

    def _fn(self, name):
        return getattr(lib(), f"fvo_{name}_{self.suf}")

    def _arr(self, a, size=None):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        if size is not None:
            assert a.size == size, (a.size, size)
        return a

    def geometry(self) -> dict:
        n = self.n
        g = dict(
            normal=np.empty(3 * 6 * n, self.dtype), normal_alt=np.empty(3 * 6 * n, self.dtype),
            area=np.empty(6 * n, self.dtype), alpha_d=np.empty(6 * n, self.dtype),
            len_c2f=np.empty(6 * n, self.dtype), volume=np.empty(n, self.dtype),
            center=np.empty(3 * n, self.dtype), is_boundary=np.empty(n, self.dtype),
            ids=np.empty(6 * n, np.int64), ids_bound_free=np.empty(6 * n, np.int64))
        self._fn("mesh_export")(self._h, *[_ptr(g[k]) for k in (
            "normal", "normal_alt", "area", "alpha_d", "len_c2f", "volume", "center", "is_boundary",
            "ids", "ids_bound_free")])
        return g

    # -- reference operators --------------------------------------------------
    def _unary(self, name, phi, mask):
        phi = self._arr(phi, self.n)
        out = np.empty(self.n, self.dtype)
        self._fn(name)(self._h, _ptr(phi), _ptr(out), int(mask))
        return out

    def grad(self, phi, mask=7):
        return self._unary("grad", phi, mask)

    def lapl(self, phi, mask=7):
        return self._unary("lapl", phi, mask)

    def stab(self, phi, mask=7):
        return self._unary("stab", phi, mask)

    def cfl_reference(self, cfl, gamma, p, rho, u, v=None, w=None):
        args = [self._arr(a, self.n) if a is not None else None for a in (p, rho, u, v, w)]
        return self._fn("cfl_reference")(self._h, float(cfl), float(gamma), *[_ptr(a) for a in args])

    # -- solvers --------------------------------------------------------------
    def heat_solve(self, T0, k, dt, steps, faithful=False):
        T = self._arr(T0, self.n).copy()
        self._fn("heat_solve")(self._h, _ptr(T), float(k), float(dt), int(steps), int(bool(faithful)))
        return T

    def heat_time(self, T0, k, dt, steps, faithful=True):
        T = self._arr(T0, self.n).copy()
        return self._fn("heat_time")(self._h, _ptr(T), float(k), float(dt), int(steps), int(bool(faithful)))

    def wave_rhs(self, q, c=None, cconst=1.0, speed_mode=0):
        q = self._arr(q, 4 * self.n)
        cc = None if c is None else self._arr(c, self.n)
        out = np.empty(4 * self.n, self.dtype)
        self._fn("wave_rhs")(self._h, _ptr(q), _ptr(cc), float(cconst), int(speed_mode), _ptr(out))
        return out

    def wave_solve(self, q0, dt, steps, c=None, cconst=1.0, speed_mode=0, faithful=False):
        q = self._arr(q0, 4 * self.n).copy()
        cc = None if c is None else self._arr(c, self.n)
        self._fn("wave_solve")(self._h, _ptr(q), _ptr(cc), float(cconst), int(speed_mode), float(dt),
                               int(steps), int(bool(faithful)))
        return q

    def wave_time(self, q0, dt, steps, cconst=1.0, faithful=True):
        q = self._arr(q0, 4 * self.n).copy()
        return self._fn("wave_time")(self._h, _ptr(q), float(cconst), float(dt), int(steps), int(bool(faithful)))

    def wave_dt(self, cfl, c=None, cconst=1.0):
        cc = None if c is None else self._arr(c, self.n)
        return self._fn("wave_dt")(self._h, _ptr(cc), float(cconst), float(cfl))

    def wave_adjoint_step(self, q, lam1, c, gc, dt):
        q = self._arr(q, 4 * self.n)
        lam1 = self._arr(lam1, 4 * self.n)
        c = self._arr(c, self.n)
        gc = self._arr(gc, self.n).copy()
        lam0 = np.empty(4 * self.n, self.dtype)
        self._fn("wave_adjoint_step")(self._h, _ptr(q), _ptr(lam1), _ptr(lam0), _ptr(c), _ptr(gc), float(dt))
        return lam0, gc

    def wave_gradient(self, q0, c, target, dt, steps):
        q0 = self._arr(q0, 4 * self.n)
        c = self._arr(c, self.n)
        target = self._arr(target, self.n)
        gc = np.empty(self.n, self.dtype)
        gp = np.empty(self.n, self.dtype)
        J = self._fn("wave_gradient")(self._h, _ptr(q0), _ptr(c), _ptr(target), float(dt), int(steps),
                                      _ptr(gc), _ptr(gp))
        return J, gc, gp

    def wave_objective(self, q0, c, target, dt, steps):
        q0 = self._arr(q0, 4 * self.n)
        c = self._arr(c, self.n)
        target = self._arr(target, self.n)
        return self._fn("wave_objective")(self._h, _ptr(q0), _ptr(c), _ptr(target), float(dt), int(steps))

    def euler_rhs(self, U, gamma=1.4):
        U = self._arr(U, 5 * self.n)
        out = np.empty(5 * self.n, self.dtype)
        self._fn("euler_rhs")(self._h, _ptr(U), float(gamma), _ptr(out))
        return out

    def euler_solve(self, U0, gamma, cfl, t_end, max_steps=1_000_000, want_totals=True):
        U = self._arr(U0, 5 * self.n).copy()
        t = np.zeros(1, np.float64)
        tot = np.zeros(2 * (max_steps + 1), np.float64) if want_totals else None
        steps = self._fn("euler_solve")(self._h, _ptr(U), float(gamma), float(cfl), float(t_end),
                                        int(max_steps), _ptr(t), _ptr(tot))
        totals = tot[: 2 * (steps + 1)].reshape(-1, 2) if want_totals else None
        return U, int(steps), float(t[0]), totals

    def total(self, f):
        return self._fn("total")(self._h, _ptr(self._arr(f, self.n)))
