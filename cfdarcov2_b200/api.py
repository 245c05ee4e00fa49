"""Thin Python front end over the C ABI for tests and the benchmark.

Device buffers are torch tensors (PyTorch is only the allocator and stream
provider here); every computation runs in libcfdb's own kernels.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import capi
from .capi import F32, F64, FUSED, PLAIN, call, lib

__all__ = ["Context", "Mesh", "Euler", "Batch", "F32", "F64", "PLAIN", "FUSED", "write_vti", "write_mesh_json",
           "save_state", "load_state"]


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _dtype_code(t) -> int:
    import torch
    if t.dtype == torch.float64:
        return F64
    if t.dtype == torch.float32:
        return F32
    raise TypeError(f"unsupported dtype {t.dtype}")


class Context:
    """cfdb_ctx bound to one CUDA device and torch's current stream on it."""

    def __init__(self, device: int = 0):
        import weakref

        import torch
        self.device = device
        self._children = weakref.WeakSet()
        self.h = C.c_void_p()
        call("cfdb_ctx_create", device, C.byref(self.h))
        self.set_stream(torch.cuda.current_stream(device).cuda_stream)

    def set_stream(self, stream_handle: int) -> None:
        call("cfdb_ctx_set_stream", self.h, C.c_void_p(stream_handle), ctx=self.h)

    def sync(self) -> None:
        call("cfdb_sync", self.h, ctx=self.h)

    def last_error(self) -> str:
        return capi.last_error(self.h)

    def set_alloc_budget(self, nbytes: int) -> None:
        call("cfdb_ctx_set_alloc_budget", self.h, int(nbytes), ctx=self.h)

    def allocated_bytes(self) -> int:
        v = C.c_int64()
        call("cfdb_ctx_allocated_bytes", self.h, C.byref(v), ctx=self.h)
        return v.value

    def launch_count(self) -> int:
        """Kernels launched on this context so far (graph replays included)."""
        v = C.c_int64()
        call("cfdb_ctx_launch_count", self.h, C.byref(v), ctx=self.h)
        return v.value

    # -- host <-> device copies through the C ABI (cfdb_upload / cfdb_download) --
    def upload(self, dst, src_host: np.ndarray | None = None, *, src_ptr=None, nbytes=None, wait=True):
        """Copies host memory into the device tensor dst; wait=False queues it
        on the context's stream (cfdb_upload_async)."""
        ptr = src_ptr if src_ptr is not None else src_host.ctypes.data
        n = nbytes if nbytes is not None else dst.numel() * dst.element_size()
        call("cfdb_upload" if wait else "cfdb_upload_async", self.h, _ptr(dst), C.c_void_p(ptr), int(n), ctx=self.h)

    def download(self, src, dst_host: np.ndarray | None = None, *, dst_ptr=None, nbytes=None, wait=True):
        """Copies the device tensor src into host memory; wait=False queues it
        on the context's stream (cfdb_download_async)."""
        ptr = dst_ptr if dst_ptr is not None else dst_host.ctypes.data
        n = nbytes if nbytes is not None else src.numel() * src.element_size()
        call("cfdb_download" if wait else "cfdb_download_async", self.h, C.c_void_p(ptr), _ptr(src), int(n),
             ctx=self.h)

    def set_wait_limit(self, cycles: int = 4000000000, missing_plane: int = -1) -> None:
        """Bound of the sweep kernels' device waits; missing_plane >= 0 is the timeout test hook."""
        call("cfdb_ctx_set_wait_limit", self.h, int(cycles), int(missing_plane), ctx=self.h)

    def trim(self) -> None:
        """Returns the workspace cached by earlier calls (checkpoint slots and
        the like) to the device."""
        call("cfdb_ctx_trim", self.h, ctx=self.h)

    def adopt(self, child) -> None:
        self._children.add(child)

    def close(self) -> None:
        if self.h:
            for child in list(self._children):
                child.close()
            lib().cfdb_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- field operators (reference operator layer) ------------------------
    def _unary_mesh_op(self, name, mesh, phi, out, mask):
        import torch
        out = torch.empty_like(phi) if out is None else out
        call(name, self.h, mesh.h, _dtype_code(phi), _ptr(phi), _ptr(out), int(mask), ctx=self.h)
        return out

    def grad(self, mesh, phi, out=None, mask=7):
        return self._unary_mesh_op("cfdb_op_grad", mesh, phi, out, mask)

    def lapl(self, mesh, phi, out=None, mask=7):
        return self._unary_mesh_op("cfdb_op_lapl", mesh, phi, out, mask)

    def stab(self, mesh, phi, out=None, mask=7):
        return self._unary_mesh_op("cfdb_op_stab", mesh, phi, out, mask)

    def binary(self, op, a, b, out=None):
        import torch
        out = torch.empty_like(a) if out is None else out
        call("cfdb_op_binary", self.h, _dtype_code(a), int(op), _ptr(a), _ptr(b), _ptr(out), a.numel(), ctx=self.h)
        return out

    def scalar(self, op, a, s, out=None):
        import torch
        out = torch.empty_like(a) if out is None else out
        call("cfdb_op_scalar", self.h, _dtype_code(a), int(op), _ptr(a), float(s), _ptr(out), a.numel(), ctx=self.h)
        return out

    def neg(self, a, out=None):
        import torch
        out = torch.empty_like(a) if out is None else out
        call("cfdb_op_neg", self.h, _dtype_code(a), _ptr(a), _ptr(out), a.numel(), ctx=self.h)
        return out

    def fill(self, out, value):
        call("cfdb_op_fill", self.h, _dtype_code(out), _ptr(out), float(value), out.numel(), ctx=self.h)
        return out

    def d1t(self, rhs, cur, dt, out=None):
        import torch
        out = torch.empty_like(cur) if out is None else out
        call("cfdb_op_d1t", self.h, _dtype_code(cur), _ptr(rhs), _ptr(cur), float(dt), _ptr(out), cur.numel(), ctx=self.h)
        return out

    def d2t(self, rhs, cur, prev, dt, second_order, out=None):
        import torch
        out = torch.empty_like(cur) if out is None else out
        call("cfdb_op_d2t", self.h, _dtype_code(cur), _ptr(rhs), _ptr(cur), _ptr(prev), float(dt), int(second_order),
             _ptr(out), cur.numel(), ctx=self.h)
        return out

    def boundary_copy(self, mesh, arr, copy, out=None):
        import torch
        out = torch.empty_like(arr) if out is None else out
        call("cfdb_op_boundary_copy", self.h, mesh.h, _dtype_code(arr), _ptr(arr), _ptr(copy), _ptr(out), ctx=self.h)
        return out

    def boundary_set_many(self, mesh, fields, values):
        """cfdb_op_boundary_set for several fields in one launch."""
        n = len(fields)
        if len(values) != n or any(t.dtype != fields[0].dtype for t in list(fields) + list(values)):
            raise ValueError("boundary_set_many: one values tensor per field, all of one dtype")
        fp = (C.c_void_p * max(n, 1))(*[t.data_ptr() for t in fields])
        vp = (C.c_void_p * max(n, 1))(*[t.data_ptr() for t in values])
        call("cfdb_op_boundary_set_many", self.h, mesh.h, _dtype_code(fields[0]) if n else F32, n, fp, vp, ctx=self.h)

    def boundary_set(self, mesh, field, values):
        """field[i] = values[i] on the boundary cells, in place."""
        call("cfdb_op_boundary_set", self.h, mesh.h, _dtype_code(field), _ptr(field), _ptr(values), ctx=self.h)
        return field

    def cfl_dt(self, mesh, cfl, gamma, p, rho, u, v=None, w=None) -> float:
        out = C.c_double()
        call("cfdb_cfl_dt", self.h, mesh.h, _dtype_code(p), float(cfl), float(gamma), _ptr(p), _ptr(rho), _ptr(u),
             _ptr(v), _ptr(w), C.byref(out), ctx=self.h)
        return out.value

    def total_fp64(self, mesh, field) -> float:
        out = C.c_double()
        call("cfdb_total_fp64", self.h, mesh.h, _dtype_code(field), _ptr(field), C.byref(out), ctx=self.h)
        return out.value

    # -- time steps -----------------------------------------------------------
    def heat_step(self, mesh, T, Tn, k, dt, path=FUSED):
        call("cfdb_heat_step", self.h, mesh.h, _dtype_code(T), int(path), _ptr(T), _ptr(Tn), float(k), float(dt),
             ctx=self.h)

    def heat_step_fixed(self, mesh, T, Tn, k, dt, fixed):
        """The fused heat step with the box-surface cells set to `fixed` in
        the same pass (cfdb_heat_step_fixed)."""
        call("cfdb_heat_step_fixed", self.h, mesh.h, _dtype_code(T), _ptr(T), _ptr(Tn), float(k), float(dt),
             _ptr(fixed), ctx=self.h)

    def d2t_step(self, mesh, u, u_prev, u_next, k, masks, dt, first_step=False):
        """One leapfrog step of d2t(u) = k * sum_j L_{masks[j]}(u), fused
        (cfdb_d2t_step): u_next = (dt dt R + 2 u) - u_prev, or dt R + u on
        the first step (u_prev unused)."""
        arr = (C.c_int32 * len(masks))(*[int(v) for v in masks])
        call("cfdb_d2t_step", self.h, mesh.h, _dtype_code(u), _ptr(u), _ptr(u_prev), _ptr(u_next), float(k), arr,
             len(masks), float(dt), int(bool(first_step)), ctx=self.h)

    def wave_step(self, mesh, q, qn, dt, c=None, c_const=1.0, speed_mode=0, path=FUSED):
        call("cfdb_wave_step", self.h, mesh.h, _dtype_code(q), int(path), _ptr(q), _ptr(qn), _ptr(c), float(c_const),
             int(speed_mode), float(dt), ctx=self.h)

    def heat_run(self, mesh, Ta, Tb, k, dt, steps, path=FUSED, use_graph=True):
        """Advances `steps` steps; returns the tensor that holds the final state."""
        fb = C.c_int()
        call("cfdb_heat_run", self.h, mesh.h, _dtype_code(Ta), int(path), _ptr(Ta), _ptr(Tb), float(k), float(dt),
             int(steps), int(bool(use_graph)), C.byref(fb), ctx=self.h)
        return Tb if fb.value else Ta

    def wave_run(self, mesh, qa, qb, dt, steps, c=None, c_const=1.0, speed_mode=0, path=FUSED, use_graph=True):
        """Advances `steps` steps; returns the tensor that holds the final state."""
        fb = C.c_int()
        call("cfdb_wave_run", self.h, mesh.h, _dtype_code(qa), int(path), _ptr(qa), _ptr(qb), _ptr(c), float(c_const),
             int(speed_mode), float(dt), int(steps), int(bool(use_graph)), C.byref(fb), ctx=self.h)
        return qb if fb.value else qa

    def wave_adjoint_step(self, mesh, q, lam1, lam0, c, gc, dt, path=FUSED):
        call("cfdb_wave_adjoint_step", self.h, mesh.h, _dtype_code(q), int(path), _ptr(q), _ptr(lam1), _ptr(lam0),
             _ptr(c), _ptr(gc), float(dt), ctx=self.h)

    def wave_gradient(self, mesh, q0, c, target, steps, dt, snapshots, grad_c, grad_p0, path=FUSED):
        J = C.c_double()
        st = capi.GradientStats()
        call("cfdb_wave_gradient", self.h, mesh.h, _dtype_code(q0), int(path), _ptr(q0), _ptr(c), _ptr(target),
             int(steps), float(dt), int(snapshots), C.byref(J), _ptr(grad_c), _ptr(grad_p0), C.byref(st), ctx=self.h)
        return J.value, st

    def wave_objective(self, mesh, q0, c, target, steps, dt, path=FUSED) -> float:
        J = C.c_double()
        call("cfdb_wave_objective", self.h, mesh.h, _dtype_code(q0), int(path), _ptr(q0), _ptr(c), _ptr(target),
             int(steps), float(dt), C.byref(J), ctx=self.h)
        return J.value


class Mesh:
    """cfdb_mesh: a structured (uniform) or vertex (distorted) hexahedral mesh."""

    def __init__(self, handle, ctx, nx, ny, nz, dx, dy, dz, uniform):
        self.h = handle
        self.ctx = ctx
        self.nx, self.ny, self.nz = nx, ny, nz
        self.n = nx * ny * nz
        self.dx, self.dy, self.dz = dx, dy, dz
        self.uniform = uniform
        if ctx is not None:
            ctx.adopt(self)

    @classmethod
    def structured(cls, ctx, nx, ny, nz, dx, dy, dz):
        h = C.c_void_p()
        call("cfdb_mesh_create_structured", ctx.h if ctx else None, nx, ny, nz, float(dx), float(dy), float(dz),
             C.byref(h), ctx=ctx.h if ctx else None)
        return cls(h, ctx, nx, ny, nz, dx, dy, dz, True)

    @classmethod
    def from_vertices(cls, ctx, nx, ny, nz, dx, dy, dz, vertices, compat_area=False):
        v = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1)
        h = C.c_void_p()
        call("cfdb_mesh_create_from_vertices", ctx.h if ctx else None, nx, ny, nz, float(dx), float(dy), float(dz),
             v.ctypes.data_as(C.c_void_p), capi.MESH_COMPAT_AREA if compat_area else 0, C.byref(h),
             ctx=ctx.h if ctx else None)
        return cls(h, ctx, nx, ny, nz, dx, dy, dz, False)

    def geometry(self, which) -> np.ndarray:
        sizes = {capi.GEOM_NORMAL: 18, capi.GEOM_NORMAL_ALT: 18, capi.GEOM_AREA: 6, capi.GEOM_ALPHA_D: 6,
                 capi.GEOM_LEN_C2F: 6, capi.GEOM_VOLUME: 1, capi.GEOM_CENTER: 3, capi.GEOM_IS_BOUNDARY: 1}
        out = np.empty(sizes[which] * self.n, np.float64)
        call("cfdb_mesh_geometry", self.h, int(which), out.ctypes.data_as(C.c_void_p),
             ctx=self.ctx.h if self.ctx else None)
        return out

    def plain_geometry(self) -> dict:
        """The FP32 face arrays the plain and generated kernels read, copied
        back from the device: ids (int32), normal, normal_alt (3 x 6n),
        area, alpha, len (6n), volume (n)."""
        g = capi.PlainGeometry()
        call("cfdb_mesh_plain_geometry", self.h, C.byref(g), ctx=self.ctx.h)
        sizes = {"ids": 6, "normal": 18, "normal_alt": 18, "area": 6, "alpha": 6, "len": 6, "volume": 1}
        out = {}
        for name, k in sizes.items():
            a = np.empty(k * self.n, np.int32 if name == "ids" else np.float32)
            call("cfdb_download", self.ctx.h, a.ctypes.data_as(C.c_void_p), C.c_void_p(getattr(g, name)),
                 a.nbytes, ctx=self.ctx.h)
            out[name] = a
        return out

    def lattice_geometry(self):
        """cfdb_mesh_lattice_geometry: (exact, constants dict)."""
        g = capi.LatticeGeometry()
        call("cfdb_mesh_lattice_geometry", self.h, C.byref(g), ctx=self.ctx.h)
        consts = {k: np.array(getattr(g, k), np.float32) for k in ("normal", "normal_alt", "area", "alpha", "len")}
        consts["volume"] = np.float32(g.volume)
        return bool(g.exact), consts

    def ids(self):
        ids = np.empty(6 * self.n, np.int64)
        ibf = np.empty(6 * self.n, np.int64)
        call("cfdb_mesh_ids", self.h, ids.ctypes.data_as(C.c_void_p), ibf.ctypes.data_as(C.c_void_p))
        return ids, ibf

    def wave_dt(self, cfl, c=None, c_const=1.0) -> float:
        out = C.c_double()
        cc = None if c is None else np.ascontiguousarray(c, dtype=np.float64)
        call("cfdb_wave_dt", self.h, None if cc is None else cc.ctypes.data_as(C.c_void_p), float(c_const),
             float(cfl), C.byref(out))
        return out.value

    def close(self):
        if self.h:
            lib().cfdb_mesh_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Euler:
    """cfdb_euler: compressible Euler with device-side dt and FP64 totals."""

    def __init__(self, ctx, mesh, dtype=F32, path=FUSED, gamma=1.4, cfl=0.4, t_end=0.2, max_steps=100000):
        self.ctx = ctx
        ctx.adopt(self)
        self.h = C.c_void_p()
        call("cfdb_euler_create", ctx.h, mesh.h, int(dtype), int(path), float(gamma), float(cfl), float(t_end),
             int(max_steps), C.byref(self.h), ctx=ctx.h)

    def begin(self, U0):
        call("cfdb_euler_begin", self.h, _ptr(U0), ctx=self.ctx.h)

    def step(self, U, Un):
        call("cfdb_euler_step", self.h, _ptr(U), _ptr(Un), ctx=self.ctx.h)

    def status(self):
        t = C.c_double()
        s = C.c_int64()
        f = C.c_int()
        call("cfdb_euler_status", self.h, C.byref(t), C.byref(s), C.byref(f), ctx=self.ctx.h)
        return t.value, s.value, bool(f.value)

    def totals(self, max_rows=200000):
        out = np.zeros(2 * max_rows, np.float64)
        rows = C.c_int64()
        call("cfdb_euler_totals", self.h, out.ctypes.data_as(C.c_void_p), int(max_rows), C.byref(rows),
             ctx=self.ctx.h)
        return out[: 2 * rows.value].reshape(-1, 2)

    def run(self, Ua, Ub, check_every=64):
        steps = C.c_int64()
        in_b = C.c_int()
        call("cfdb_euler_run", self.h, _ptr(Ua), _ptr(Ub), int(check_every), C.byref(steps), C.byref(in_b),
             ctx=self.ctx.h)
        return steps.value, bool(in_b.value)

    def close(self):
        if self.h:
            lib().cfdb_euler_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """cfdb_batch: an ensemble of independent cubes advanced together."""

    def __init__(self, ctx, problems):
        self.ctx = ctx
        ctx.adopt(self)
        arr = (capi.Problem * len(problems))()
        for i, p in enumerate(problems):
            arr[i].n, arr[i].kind, arr[i].param, arr[i].dt = int(p["n"]), int(p["kind"]), float(p["param"]), float(p["dt"])
        self.h = C.c_void_p()
        pool = C.c_int64()
        call("cfdb_batch_create", ctx.h, arr, len(problems), C.byref(pool), C.byref(self.h), ctx=ctx.h)
        self.pool_elems = pool.value
        self.offsets = [arr[i].offset for i in range(len(problems))]

    def set_config(self, cells_per_item, threads, ctas_per_sm):
        call("cfdb_batch_set_config", self.h, int(cells_per_item), int(threads), int(ctas_per_sm), ctx=self.ctx.h)

    def set_staged(self, form) -> None:
        """Kernel form: 0 / False column march, 1 / True staged row ring, 2 column march at 48 registers."""
        call("cfdb_batch_set_staged", self.h, int(form), ctx=self.ctx.h)

    def get_config(self):
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        call("cfdb_batch_get_config", self.h, C.byref(a), C.byref(b), C.byref(c), ctx=self.ctx.h)
        return a.value, b.value, c.value

    def tune(self, pool_a, pool_b, cache_path=None):
        call("cfdb_batch_tune", self.h, _ptr(pool_a), _ptr(pool_b),
             None if cache_path is None else str(cache_path).encode(), ctx=self.ctx.h)

    def step(self, a, b):
        call("cfdb_batch_step", self.h, _ptr(a), _ptr(b), ctx=self.ctx.h)

    def run(self, a, b, steps, use_graph=True):
        """Advances `steps` steps a -> b -> a ...; returns the pool that holds the final state."""
        call("cfdb_batch_run", self.h, _ptr(a), _ptr(b), int(steps), int(bool(use_graph)), ctx=self.ctx.h)
        return a if steps % 2 == 0 else b

    def launch_count(self) -> int:
        v = C.c_int64()
        call("cfdb_batch_launch_count", self.h, C.byref(v), ctx=self.ctx.h)
        return v.value

    def close(self):
        if self.h:
            lib().cfdb_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def revolve_plan(steps: int, snapshots: int):
    """Binomial checkpointing schedule as a list of (action, arg, step)."""
    count = C.c_int64()
    fwd = C.c_int64()
    call("cfdb_revolve_plan", int(steps), int(snapshots), None, None, None, 0, C.byref(count), C.byref(fwd))
    n = count.value
    a = np.zeros(n, np.int32)
    g = np.zeros(n, np.int32)
    s = np.zeros(n, np.int32)
    call("cfdb_revolve_plan", int(steps), int(snapshots), a.ctypes.data_as(C.c_void_p), g.ctypes.data_as(C.c_void_p),
         s.ctypes.data_as(C.c_void_p), n, C.byref(count), C.byref(fwd))
    return list(zip(a.tolist(), g.tolist(), s.tolist())), fwd.value


def write_vti(path, name, values, nx, ny, nz):
    """VTK image (.vti) of a field given in cell order (z fastest), as the
    reference's store_history writes it; `values` is host data (numpy or a
    CPU tensor), converted to float32."""
    v = np.ascontiguousarray(np.asarray(values, dtype=np.float32).reshape(-1))
    if v.size != nx * ny * nz:
        raise ValueError("values do not match the mesh size")
    call("cfdb_write_vti", os.fsencode(path), str(name).encode(), int(nx), int(ny), int(nz),
         v.ctypes.data_as(C.c_void_p))


def write_mesh_json(path, nx, ny, nz, dx, dy, dz, vertices=None):
    """mesh.json as the reference's store_mesh writes it."""
    ptr = None
    if vertices is not None:
        vertices = np.ascontiguousarray(np.asarray(vertices, dtype=np.float64).reshape(-1))
        if vertices.size != 3 * (nx + 1) * (ny + 1) * (nz + 1):
            raise ValueError("vertices do not match the mesh size")
        ptr = vertices.ctypes.data_as(C.c_void_p)
    call("cfdb_write_mesh_json", os.fsencode(path), int(nx), int(ny), int(nz), float(dx), float(dy), float(dz), ptr)


def save_state(path, values, nx, ny, nz, fields, step=0, t=0.0):
    """Checkpoint (cfdb_state_save) of host data holding `fields` x n values
    in field order; float32 or float64 as given."""
    v = np.ascontiguousarray(np.asarray(values).reshape(-1))
    if v.dtype not in (np.float32, np.float64) or v.size != fields * nx * ny * nz:
        raise ValueError("values must be float32 or float64 with fields x nx x ny x nz entries")
    call("cfdb_state_save", os.fsencode(path), F64 if v.dtype == np.float64 else F32, int(nx), int(ny), int(nz),
         int(fields), int(step), float(t), v.ctypes.data_as(C.c_void_p))


def load_state(path, nx, ny, nz, fields, dtype=np.float32):
    """(values, step, t) of a checkpoint written by save_state; the dtype,
    dimensions and field count must match the file's."""
    dt = np.dtype(dtype)
    out = np.empty(fields * nx * ny * nz, dt)
    step, t = C.c_int64(), C.c_double()
    call("cfdb_state_load", os.fsencode(path), F64 if dt == np.float64 else F32, int(nx), int(ny), int(nz),
         int(fields), C.byref(step), C.byref(t), out.ctypes.data_as(C.c_void_p))
    return out, step.value, t.value
