// Plain (per-operator) kernels over the reference's N x 6 geometry arrays, in
// float and double: the B200 replacement of src/cuda_operators.cu.  Each
// kernel writes into a caller buffer (no allocation per call, no device-wide
// sync).  This file is compiled with --fmad=false and IEEE division / square
// root so that every multiply and add rounds separately, in the same order as
// the CPU oracle; the FP64 path then matches the FP64 oracle bit for bit.
//
// Face sums run over slots 0..5 in order, per dimension, as the reference's
// device helper gauss_grad_cu_k does (include/custom_cuda_functions.hpp:147-162).
#include <cmath>

#include "cfdb_internal.hpp"

CFDB_MODULE_ANCHOR

namespace {

constexpr int kThreads = 256;

template <class R> struct PlainArgs {
  const int32_t* __restrict__ ids;
  const R* __restrict__ normal;      // 3 x 6n
  const R* __restrict__ normal_alt;  // 3 x 6n
  const R* __restrict__ area;
  const R* __restrict__ alpha;
  const R* __restrict__ len;
  const R* __restrict__ volume;
  const R* __restrict__ isb;
  int64_t n;
};

template <class R> PlainArgs<R> plain_args(const cfdb_mesh* m, int dtype) {
  const PlainGeomDev& p = m->plain[dtype == CFDB_F64 ? 1 : 0];
  PlainArgs<R> a;
  a.ids = m->d_ids;
  a.normal = static_cast<const R*>(p.normal);
  a.normal_alt = static_cast<const R*>(p.normal_alt);
  a.area = static_cast<const R*>(p.area);
  a.alpha = static_cast<const R*>(p.alpha);
  a.len = static_cast<const R*>(p.len);
  a.volume = static_cast<const R*>(p.volume);
  a.isb = static_cast<const R*>(p.isb);
  a.n = m->n;
  return a;
}

#define GRID_STRIDE(i, n) for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < (n); i += int64_t(gridDim.x) * blockDim.x)

// GradVar / eval_grad_k (src/cuda_operators.cu:237-283).
template <class R> __global__ void grad_k(PlainArgs<R> g, const R* __restrict__ phi, R* __restrict__ out, int mask) {
  const int64_t n = g.n;
  GRID_STRIDE(i, n) {
    const R crr = phi[i];
    R res = R(0);
    for (int d = 0; d < 3; ++d) {
      R acc = R(0);
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const int64_t k6 = int64_t(f) * n + i;
        const R itp = (crr + phi[g.ids[k6]]) * R(0.5);
        const R t = itp * g.normal_alt[int64_t(d) * 6 * n + k6];
        acc = acc + t * g.area[k6];
      }
      const R gd = acc / g.volume[i];
      if (mask & (1 << d)) res = res + gd;
    }
    out[i] = res;
  }
}

// Grad2Var / eval_grad2_k (src/cuda_operators.cu:490-544).
template <class R> __device__ __forceinline__ R lapl_at(const PlainArgs<R>& g, const R* __restrict__ phi, int64_t i, int mask) {
  const int64_t n = g.n;
  const R crr = phi[i];
  R sn[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const int64_t k6 = int64_t(f) * n + i;
    sn[f] = (phi[g.ids[k6]] - crr) * g.alpha[k6];
  }
  R res = R(0);
  for (int d = 0; d < 3; ++d) {
    if (!(mask & (1 << d))) continue;
    R acc = R(0);
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const int64_t k6 = int64_t(f) * n + i;
      const R t = sn[f] * g.normal[int64_t(d) * 6 * n + k6];
      acc = acc + t * g.area[k6];
    }
    res = res + acc / g.volume[i];
  }
  return res;
}

template <class R> __global__ void lapl_k(PlainArgs<R> g, const R* __restrict__ phi, R* __restrict__ out, int mask) {
  GRID_STRIDE(i, g.n) out[i] = lapl_at(g, phi, i, mask);
}

// StabVar stage 1 / stage 2 (src/cuda_operators.cu:307-434).
template <class R> __global__ void stab1_k(PlainArgs<R> g, const R* __restrict__ phi, R* __restrict__ up) {
  const int64_t n = g.n;
  GRID_STRIDE(i, n) {
    const R crr = phi[i];
    R gr[3];
    for (int d = 0; d < 3; ++d) {
      R acc = R(0);
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const int64_t k6 = int64_t(f) * n + i;
        const R itp = (crr + phi[g.ids[k6]]) * R(0.5);
        const R t = itp * g.normal_alt[int64_t(d) * 6 * n + k6];
        acc = acc + t * g.area[k6];
      }
      gr[d] = acc / g.volume[i];
    }
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const int64_t k6 = int64_t(f) * n + i;
        const int64_t kd = int64_t(d) * 6 * n + k6;
        up[kd] = crr + g.len[k6] * gr[d] * g.normal_alt[kd];
      }
  }
}

template <class R> __global__ void stab2_k(PlainArgs<R> g, const R* __restrict__ up, R* __restrict__ out, int mask) {
  const int64_t n = g.n;
  GRID_STRIDE(i, n) {
    R res = R(0);
    for (int d = 0; d < 3; ++d) {
      if (!(mask & (1 << d))) continue;
      const R* u = up + int64_t(d) * 6 * n;
      R acc = R(0);
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const int64_t k6 = int64_t(f) * n + i;
        const R col = u[int64_t(f ^ 1) * n + g.ids[k6]];
        const R s = R(0.5) * (u[k6] - col);
        const R t = s * g.normal[int64_t(d) * 6 * n + k6];
        acc = acc + t * g.area[k6];
      }
      res = res + acc / g.volume[i];
    }
    out[i] = res;
  }
}

// ---- elementwise (src/cuda_operators.cu:27-136) --------------------------
template <class R> __global__ void binary_k(int op, const R* __restrict__ a, const R* __restrict__ b, R* __restrict__ c, int64_t n) {
  GRID_STRIDE(i, n) {
    const R x = a[i], y = b[i];
    R r;
    switch (op) {
      case CFDB_OP_ADD: r = x + y; break;
      case CFDB_OP_SUB: r = x - y; break;
      case CFDB_OP_MUL: r = x * y; break;
      default: r = x / y; break;
    }
    c[i] = r;
  }
}

template <class R> __global__ void scalar_k(int op, const R* __restrict__ a, R s, R* __restrict__ c, int64_t n) {
  GRID_STRIDE(i, n) {
    const R x = a[i];
    R r;
    switch (op) {
      case CFDB_OP_ADD: r = x + s; break;
      case CFDB_OP_SUB: r = x - s; break;
      case CFDB_OP_MUL: r = x * s; break;
      case CFDB_OP_DIV: r = x / s; break;
      case CFDB_OP_RSUB: r = s - x; break;
      default: r = s / x; break;
    }
    c[i] = r;
  }
}

template <class R> __global__ void neg_k(const R* __restrict__ a, R* __restrict__ c, int64_t n) { GRID_STRIDE(i, n) c[i] = -a[i]; }
template <class R> __global__ void fill_k(R* __restrict__ c, R v, int64_t n) { GRID_STRIDE(i, n) c[i] = v; }

// DtVar: next = dt * rhs + cur (src/fvm3d.cpp:690-697).
template <class R> __global__ void d1t_k(const R* __restrict__ rhs, const R* __restrict__ cur, R dt, R* __restrict__ nxt, int64_t n) {
  GRID_STRIDE(i, n) nxt[i] = dt * rhs[i] + cur[i];
}

// D2tVar: next = dt*dt*rhs + 2*cur - prev (src/fvm3d.cpp:735-751).
template <class R> __global__ void d2t_k(const R* __restrict__ rhs, const R* __restrict__ cur, const R* __restrict__ prev, R dt, int second,
                                         R* __restrict__ nxt, int64_t n) {
  GRID_STRIDE(i, n) {
    if (second) nxt[i] = (dt * dt * rhs[i] + R(2) * cur[i]) - prev[i];
    else nxt[i] = dt * rhs[i] + cur[i];
  }
}

// heat update T' = dt * (k * L) + T (the reference's 3.0 * lapl(T) then DtVar).
template <class R> __global__ void heat_update_k(const R* __restrict__ L, const R* __restrict__ T, R k, R dt, R* __restrict__ Tn, int64_t n) {
  GRID_STRIDE(i, n) {
    const R rhs = k * L[i];
    Tn[i] = dt * rhs + T[i];
  }
}

// _boundary_copy_cu (examples/main_3d_heat.cpp:41-46).
template <class R> __global__ void bcopy_k(const R* __restrict__ arr, const R* __restrict__ cp, const R* __restrict__ isb, R* __restrict__ out, int64_t n) {
  GRID_STRIDE(i, n) {
    const R b = isb[i];
    out[i] = arr[i] * (R(1) - b) + cp[i] * b;
  }
}

// the cells of the box surface: the two x planes (all y, z), the two y planes
// and the two z planes; cells on edges and corners come up more than once and
// are written with the same value each time
template <class R>
__global__ void bset_k(R* __restrict__ field, const R* __restrict__ values, int64_t nx, int64_t ny, int64_t nz) {
  const int64_t px = ny * nz, py = nx * nz, pz = nx * ny, total = 2 * (px + py + pz);
  GRID_STRIDE(t, total) {
    int64_t x, y, z;
    if (t < 2 * px) {
      const int64_t r = t % px;
      x = t < px ? 0 : nx - 1, y = r / nz, z = r % nz;
    } else if (t < 2 * (px + py)) {
      const int64_t u = t - 2 * px, r = u % py;
      y = u < py ? 0 : ny - 1, x = r / nz, z = r % nz;
    } else {
      const int64_t u = t - 2 * (px + py), r = u % pz;
      z = u < pz ? 0 : nz - 1, x = r / ny, y = r % ny;
    }
    const int64_t i = (x * ny + y) * nz + z;
    field[i] = values[i];
  }
}

// bset_k for up to kSetBatch fields in one launch: field k = blockIdx.y
constexpr int kSetBatch = 16;
template <class R> struct SetBatch {
  R* field[kSetBatch];
  const R* values[kSetBatch];
};
template <class R>
__global__ void bset_many_k(SetBatch<R> b, int64_t nx, int64_t ny, int64_t nz) {
  R* __restrict__ field = b.field[blockIdx.y];
  const R* __restrict__ values = b.values[blockIdx.y];
  const int64_t px = ny * nz, py = nx * nz, pz = nx * ny, total = 2 * (px + py + pz);
  GRID_STRIDE(t, total) {
    int64_t x, y, z;
    if (t < 2 * px) {
      const int64_t r = t % px;
      x = t < px ? 0 : nx - 1, y = r / nz, z = r % nz;
    } else if (t < 2 * (px + py)) {
      const int64_t u = t - 2 * px, r = u % py;
      y = u < py ? 0 : ny - 1, x = r / nz, z = r % nz;
    } else {
      const int64_t u = t - 2 * (px + py), r = u % pz;
      z = u < pz ? 0 : nz - 1, x = r / ny, y = r % ny;
    }
    const int64_t i = (x * ny + y) * nz + z;
    field[i] = values[i];
  }
}

// ---- reductions -------------------------------------------------------------
__device__ __forceinline__ void atomic_min_pos(float* a, float v) { atomicMin(reinterpret_cast<int*>(a), __float_as_int(v)); }
__device__ __forceinline__ void atomic_min_pos(double* a, double v) {
  atomicMin(reinterpret_cast<unsigned long long*>(a), static_cast<unsigned long long>(__double_as_longlong(v)));
}

// cfl_cu_k + thrust::min_element (src/cuda_operators.cu:138-235).
template <class R>
__global__ void cfl_k(R dl, R gamma, const R* __restrict__ p, const R* __restrict__ rho, const R* __restrict__ u,
                      const R* __restrict__ v, const R* __restrict__ w, int64_t n, R* __restrict__ result) {
  __shared__ R red[kThreads / 32];
  R best = R(INFINITY);
  GRID_STRIDE(i, n) {
    R vv = u[i] * u[i];
    if (v) vv = vv + v[i] * v[i];
    if (w) vv = vv + w[i] * w[i];
    const R den = dl * (R(1) / (sqrt((gamma * p[i]) / rho[i]) + sqrt(vv)));
    best = fmin(best, den);
  }
  for (int o = 16; o > 0; o >>= 1) best = fmin(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x < 32) {
    best = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : R(INFINITY);
    for (int o = 16; o > 0; o >>= 1) best = fmin(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (threadIdx.x == 0) atomic_min_pos(result, best);
  }
}

// Neumaier (compensated) accumulation of field * V in double.
struct Comp { double s, c; };
__device__ __forceinline__ void comp_add(Comp& a, double x) {
  const double t = a.s + x;
  if (fabs(a.s) >= fabs(x)) a.c += (a.s - t) + x; else a.c += (x - t) + a.s;
  a.s = t;
}
__device__ __forceinline__ void comp_merge(Comp& a, Comp b) {
  comp_add(a, b.s);
  a.c += b.c;
}

template <class R>
__global__ void total_k(const R* __restrict__ f, const R* __restrict__ vol, double vconst, int64_t n, Comp* __restrict__ part) {
  __shared__ Comp red[kThreads / 32];
  Comp a{0.0, 0.0};
  GRID_STRIDE(i, n) comp_add(a, double(f[i]) * (vol ? double(vol[i]) : vconst));
  for (int o = 16; o > 0; o >>= 1) {
    Comp b{__shfl_xor_sync(0xffffffffu, a.s, o), __shfl_xor_sync(0xffffffffu, a.c, o)};
    comp_merge(a, b);
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    Comp t{0.0, 0.0};
    for (int w = 0; w < int(blockDim.x / 32); ++w) comp_merge(t, red[w]);
    part[blockIdx.x] = t;
  }
}

__global__ void total_final_k(const Comp* __restrict__ part, int np, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    Comp t{0.0, 0.0};
    for (int k = 0; k < np; ++k) comp_merge(t, part[k]);
    out[0] = t.s + t.c;
  }
}

// ---- the acoustic system on the general geometry ------------------------------
// Same arithmetic as the CPU oracle's wave_rhs_cell followed by the DtVar update.
template <class R>
__global__ void wave_plain_k(PlainArgs<R> g, const R* __restrict__ q, R* __restrict__ qn, const R* __restrict__ cf, R cconst,
                             int mode, R dt) {
  const int64_t n = g.n;
  GRID_STRIDE(i, n) {
    const R pP = q[i], uP = q[n + i], vP = q[2 * n + i], wP = q[3 * n + i];
    const R cP = cf ? cf[i] : cconst;
    const R c2 = cP * cP;
    R ap = R(0), au = R(0), av = R(0), aw = R(0);
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const int64_t k6 = int64_t(f) * n + i;
      const R nx = g.normal_alt[k6], ny = g.normal_alt[6 * n + k6], nz = g.normal_alt[12 * n + k6];
      const R A = g.area[k6];
      const R unP = (uP * nx + vP * ny) + wP * nz;
      const int64_t j = g.ids[k6];
      R pN, uN, vN, wN, cN;
      if (j != i) {
        pN = q[j]; uN = q[n + j]; vN = q[2 * n + j]; wN = q[3 * n + j];
        cN = cf ? cf[j] : cconst;
      } else {
        const R two_un = R(2) * unP;
        pN = pP; uN = uP - two_un * nx; vN = vP - two_un * ny; wN = wP - two_un * nz; cN = cP;
      }
      const R unN = (uN * nx + vN * ny) + wN * nz;
      const R cfc = mode == 0 ? fmax(cP, cN) : R(0.5) * (cP + cN);
      const R hc = R(0.5) * cfc;
      const R fp = c2 * (R(0.5) * (unP + unN)) - hc * (pN - pP);
      const R pm = R(0.5) * (pP + pN);
      const R fu = pm * nx - hc * (uN - uP);
      const R fv = pm * ny - hc * (vN - vP);
      const R fw = pm * nz - hc * (wN - wP);
      ap = ap + fp * A; au = au + fu * A; av = av + fv * A; aw = aw + fw * A;
    }
    const R V = g.volume[i];
    qn[i] = dt * (-(ap / V)) + pP;
    qn[n + i] = dt * (-(au / V)) + uP;
    qn[2 * n + i] = dt * (-(av / V)) + vP;
    qn[3 * n + i] = dt * (-(aw / V)) + wP;
  }
}

// Adjoint of wave_plain_k for mode 1, same arithmetic as the oracle's
// wave_adjoint_step (volume-scaled adjoint lt = lam / V).
template <class R>
__global__ void wave_adjoint_plain_k(PlainArgs<R> g, const R* __restrict__ q, const R* __restrict__ lam1, R* __restrict__ lam0,
                                     const R* __restrict__ cf, R* __restrict__ gc, R dt) {
  const int64_t n = g.n;
  GRID_STRIDE(i, n) {
    const R cP = cf[i];
    const R iVP = R(1) / g.volume[i];
    const R lpP = lam1[i] * iVP, luP = lam1[n + i] * iVP, lvP = lam1[2 * n + i] * iVP, lwP = lam1[3 * n + i] * iVP;
    const R pP = q[i], uP = q[n + i], vP = q[2 * n + i], wP = q[3 * n + i];
    R ap = R(0), au = R(0), av = R(0), aw = R(0), gg = R(0);
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const int64_t k6 = int64_t(f) * n + i;
      const R nx = g.normal_alt[k6], ny = g.normal_alt[6 * n + k6], nz = g.normal_alt[12 * n + k6];
      const R A = g.area[k6];
      const R Sx = nx * A, Sy = ny * A, Sz = nz * A;
      const int64_t j = g.ids[k6];
      if (j != i) {
        const R cN = cf[j];
        const R iVN = R(1) / g.volume[j];
        const R h = R(0.5) * (R(0.5) * (cP + cN)) * A;
        const R lpN = lam1[j] * iVN, luN = lam1[n + j] * iVN, lvN = lam1[2 * n + j] * iVN, lwN = lam1[3 * n + j] * iVN;
        const R Slu_d = (Sx * (luN - luP) + Sy * (lvN - lvP)) + Sz * (lwN - lwP);
        ap = ap + (h * (lpN - lpP) + R(0.5) * Slu_d);
        const R sp = R(0.5) * (cN * cN * lpN - cP * cP * lpP);
        au = au + (sp * Sx + h * (luN - luP));
        av = av + (sp * Sy + h * (lvN - lvP));
        aw = aw + (sp * Sz + h * (lwN - lwP));
        const R pN = q[j], uN = q[n + j], vN = q[2 * n + j], wN = q[3 * n + j];
        const R Su_sum = (Sx * (uP + uN) + Sy * (vP + vN)) + Sz * (wP + wN);
        gg = gg - cP * Su_sum * lpP;
        const R jp = pN - pP;
        const R ju_self = ((uN - uP) * luP + (vN - vP) * lvP) + (wN - wP) * lwP;
        const R ju_nb = ((uP - uN) * luN + (vP - vN) * lvN) + (wP - wN) * lwN;
        gg = gg + R(0.25) * A * ((jp * lpP + ju_self) + (ju_nb - jp * lpN));
      } else {
        const R Slu = (Sx * luP + Sy * lvP) + Sz * lwP;
        ap = ap - Slu;
        const R lun = (luP * nx + lvP * ny) + lwP * nz;
        const R cA = cP * A;
        au = au - cA * lun * nx; av = av - cA * lun * ny; aw = aw - cA * lun * nz;
        const R un = (uP * nx + vP * ny) + wP * nz;
        gg = gg - A * un * lun;
      }
    }
    lam0[i] = lam1[i] + dt * ap;
    lam0[n + i] = lam1[n + i] + dt * au;
    lam0[2 * n + i] = lam1[2 * n + i] + dt * av;
    lam0[3 * n + i] = lam1[3 * n + i] + dt * aw;
    gc[i] = gc[i] + dt * gg;
  }
}

int need(cfdb_ctx* ctx, cfdb_mesh* m, int dtype) {
  if (int rc = cfdb_check_mesh(ctx, m)) return rc;
  if (!dtype_ok(dtype)) return cfdb_fail(ctx, CFDB_EINVAL, "unknown dtype %d", dtype);
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  return cfdb_mesh_need_plain(m, dtype);
}

int check_ptrs(cfdb_ctx* ctx, const char* fn, std::initializer_list<const void*> ps) {
  for (const void* p : ps)
    if (!p) return cfdb_fail(ctx, CFDB_EINVAL, "%s: NULL field pointer", fn);
  return CFDB_OK;
}

int check_n(cfdb_ctx* ctx, int dtype, int64_t n, const char* fn) {
  if (!ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "%s: ctx is NULL", fn);
  if (!dtype_ok(dtype)) return cfdb_fail(ctx, CFDB_EINVAL, "%s: unknown dtype %d", fn, dtype);
  if (n < 0) return cfdb_fail(ctx, CFDB_EINVAL, "%s: negative length", fn);
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  return CFDB_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// entry points
// ---------------------------------------------------------------------------
#define DISPATCH(dtype, R, ...)          \
  if ((dtype) == CFDB_F64) {             \
    using R = double;                    \
    __VA_ARGS__;                         \
  } else {                               \
    using R = float;                     \
    __VA_ARGS__;                         \
  }

extern "C" int cfdb_op_grad(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* phi, void* out, int mask) {
  if (int rc = need(ctx, m, dtype)) return rc;
  if (int rc = check_ptrs(ctx, "cfdb_op_grad", {phi, out})) return rc;
  if (mask < 0 || mask > 7) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_op_grad: dims_mask %d out of range", mask);
  const int grid = grid_for(ctx, m->n, kThreads);
  DISPATCH(dtype, R, grad_k<R><<<grid, kThreads, 0, ctx->stream>>>(plain_args<R>(m, dtype), (const R*)phi, (R*)out, mask));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}

int plain_lapl(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* phi, void* out, int mask) {
  const int grid = grid_for(ctx, m->n, kThreads);
  DISPATCH(dtype, R, lapl_k<R><<<grid, kThreads, 0, ctx->stream>>>(plain_args<R>(m, dtype), (const R*)phi, (R*)out, mask));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}

extern "C" int cfdb_op_lapl(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* phi, void* out, int mask) {
  if (int rc = need(ctx, m, dtype)) return rc;
  if (int rc = check_ptrs(ctx, "cfdb_op_lapl", {phi, out})) return rc;
  if (mask < 0 || mask > 7) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_op_lapl: dims_mask %d out of range", mask);
  return plain_lapl(ctx, m, dtype, phi, out, mask);
}

extern "C" int cfdb_op_stab(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* phi, void* out, int mask) {
  if (int rc = need(ctx, m, dtype)) return rc;
  if (int rc = check_ptrs(ctx, "cfdb_op_stab", {phi, out})) return rc;
  if (mask < 0 || mask > 7) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_op_stab: dims_mask %d out of range", mask);
  PlainGeomDev& p = m->plain[dtype == CFDB_F64 ? 1 : 0];
  if (!p.stab_tmp)
    if (int rc = cfdb_dev_alloc(ctx, int64_t(dtype_size(dtype)) * 18 * m->n, &p.stab_tmp)) return rc;
  const int grid = grid_for(ctx, m->n, kThreads);
  DISPATCH(dtype, R, {
    stab1_k<R><<<grid, kThreads, 0, ctx->stream>>>(plain_args<R>(m, dtype), (const R*)phi, (R*)p.stab_tmp);
    stab2_k<R><<<grid, kThreads, 0, ctx->stream>>>(plain_args<R>(m, dtype), (const R*)p.stab_tmp, (R*)out, mask);
  });
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}

extern "C" int cfdb_op_binary(cfdb_ctx* ctx, int dtype, int op, const void* a, const void* b, void* out, int64_t n) {
  if (int rc = check_n(ctx, dtype, n, "cfdb_op_binary")) return rc;
  if (op < CFDB_OP_ADD || op > CFDB_OP_DIV) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_op_binary: bad op %d", op);
  if (n == 0) return CFDB_OK;
  if (int rc = check_ptrs(ctx, "cfdb_op_binary", {a, b, out})) return rc;
  DISPATCH(dtype, R, binary_k<R><<<grid_for(ctx, n, kThreads), kThreads, 0, ctx->stream>>>(op, (const R*)a, (const R*)b, (R*)out, n));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}

extern "C" int cfdb_op_scalar(cfdb_ctx* ctx, int dtype, int op, const void* a, double s, void* out, int64_t n) {
  if (int rc = check_n(ctx, dtype, n, "cfdb_op_scalar")) return rc;
  if (op < CFDB_OP_ADD || op > CFDB_OP_RDIV) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_op_scalar: bad op %d", op);
  if (n == 0) return CFDB_OK;
  if (int rc = check_ptrs(ctx, "cfdb_op_scalar", {a, out})) return rc;
  DISPATCH(dtype, R, scalar_k<R><<<grid_for(ctx, n, kThreads), kThreads, 0, ctx->stream>>>(op, (const R*)a, R(s), (R*)out, n));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}

extern "C" int cfdb_op_neg(cfdb_ctx* ctx, int dtype, const void* a, void* out, int64_t n) {
  if (int rc = check_n(ctx, dtype, n, "cfdb_op_neg")) return rc;
  if (n == 0) return CFDB_OK;
  if (int rc = check_ptrs(ctx, "cfdb_op_neg", {a, out})) return rc;
  DISPATCH(dtype, R, neg_k<R><<<grid_for(ctx, n, kThreads), kThreads, 0, ctx->stream>>>((const R*)a, (R*)out, n));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}

extern "C" int cfdb_op_fill(cfdb_ctx* ctx, int dtype, void* out, double value, int64_t n) {
  if (int rc = check_n(ctx, dtype, n, "cfdb_op_fill")) return rc;
  if (n == 0) return CFDB_OK;
  if (int rc = check_ptrs(ctx, "cfdb_op_fill", {out})) return rc;
  DISPATCH(dtype, R, fill_k<R><<<grid_for(ctx, n, kThreads), kThreads, 0, ctx->stream>>>((R*)out, R(value), n));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}

extern "C" int cfdb_op_d1t(cfdb_ctx* ctx, int dtype, const void* rhs, const void* cur, double dt, void* next, int64_t n) {
  if (int rc = check_n(ctx, dtype, n, "cfdb_op_d1t")) return rc;
  if (n == 0) return CFDB_OK;
  if (int rc = check_ptrs(ctx, "cfdb_op_d1t", {rhs, cur, next})) return rc;
  DISPATCH(dtype, R, d1t_k<R><<<grid_for(ctx, n, kThreads), kThreads, 0, ctx->stream>>>((const R*)rhs, (const R*)cur, R(dt), (R*)next, n));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}

extern "C" int cfdb_op_d2t(cfdb_ctx* ctx, int dtype, const void* rhs, const void* cur, const void* prev, double dt,
                           int second_order, void* next, int64_t n) {
  if (int rc = check_n(ctx, dtype, n, "cfdb_op_d2t")) return rc;
  if (n == 0) return CFDB_OK;
  if (int rc = check_ptrs(ctx, "cfdb_op_d2t", {rhs, cur, next})) return rc;
  if (second_order && !prev) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_op_d2t: prev is NULL for a second-order step");
  DISPATCH(dtype, R, d2t_k<R><<<grid_for(ctx, n, kThreads), kThreads, 0, ctx->stream>>>((const R*)rhs, (const R*)cur, (const R*)prev, R(dt), second_order, (R*)next, n));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}

int plain_heat_update(cfdb_ctx* ctx, int dtype, const void* L, const void* T, double k, double dt, void* Tn, int64_t n) {
  DISPATCH(dtype, R, heat_update_k<R><<<grid_for(ctx, n, kThreads), kThreads, 0, ctx->stream>>>((const R*)L, (const R*)T, R(k), R(dt), (R*)Tn, n));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}

extern "C" int cfdb_op_boundary_copy(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* arr, const void* cp, void* out) {
  if (int rc = need(ctx, m, dtype)) return rc;
  if (int rc = check_ptrs(ctx, "cfdb_op_boundary_copy", {arr, cp, out})) return rc;
  const PlainGeomDev& p = m->plain[dtype == CFDB_F64 ? 1 : 0];
  DISPATCH(dtype, R, bcopy_k<R><<<grid_for(ctx, m->n, kThreads), kThreads, 0, ctx->stream>>>((const R*)arr, (const R*)cp, (const R*)p.isb, (R*)out, m->n));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}

extern "C" int cfdb_op_boundary_set(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, void* field, const void* values) {
  if (int rc = cfdb_check_mesh(ctx, m)) return rc;
  if (!dtype_ok(dtype)) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_op_boundary_set: unknown dtype %d", dtype);
  if (int rc = check_ptrs(ctx, "cfdb_op_boundary_set", {field, values})) return rc;
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  const int64_t total = 2 * (m->ny * m->nz + m->nx * m->nz + m->nx * m->ny);
  DISPATCH(dtype, R, bset_k<R><<<grid_for(ctx, total, kThreads), kThreads, 0, ctx->stream>>>((R*)field, (const R*)values, m->nx, m->ny, m->nz));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}

extern "C" int cfdb_op_boundary_set_many(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, int32_t count, void* const* fields,
                                         const void* const* values) {
  if (int rc = cfdb_check_mesh(ctx, m)) return rc;
  if (!dtype_ok(dtype)) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_op_boundary_set_many: unknown dtype %d", dtype);
  if (count < 0 || (count > 0 && (!fields || !values)))
    return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_op_boundary_set_many: bad field list");
  for (int32_t k = 0; k < count; ++k)
    if (int rc = check_ptrs(ctx, "cfdb_op_boundary_set_many", {fields[k], values[k]})) return rc;
  if (count == 0) return CFDB_OK;
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  const int64_t total = 2 * (m->ny * m->nz + m->nx * m->nz + m->nx * m->ny);
  for (int32_t k0 = 0; k0 < count; k0 += kSetBatch) {
    const int nb = std::min<int32_t>(kSetBatch, count - k0);
    // one CTA row per field; the fields share the launch's x extent
    const dim3 grid(unsigned(std::max(1, grid_for(ctx, total, kThreads) / nb)), unsigned(nb));
    DISPATCH(dtype, R, {
      SetBatch<R> b{};
      for (int j = 0; j < nb; ++j) {
        b.field[j] = static_cast<R*>(fields[k0 + j]);
        b.values[j] = static_cast<const R*>(values[k0 + j]);
      }
      bset_many_k<R><<<grid, kThreads, 0, ctx->stream>>>(b, m->nx, m->ny, m->nz);
    });
    CFDB_LAUNCHED(ctx);
  }
  return CFDB_OK;
}

extern "C" int cfdb_cfl_dt(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, double cfl, double gamma, const void* p,
                           const void* rho, const void* u, const void* v, const void* w, double* dt_out) {
  if (int rc = cfdb_check_mesh(ctx, m)) return rc;
  if (!dtype_ok(dtype)) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_cfl_dt: unknown dtype %d", dtype);
  if (int rc = check_ptrs(ctx, "cfdb_cfl_dt", {p, rho, u, dt_out})) return rc;
  if ((v == nullptr) != (w == nullptr)) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_cfl_dt: give both v and w or neither");
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  void* res = nullptr;
  if (int rc = cfdb_ws_alloc(ctx, 8, &res)) return rc;
  int rc = CFDB_OK;
  double host = 0;
  DISPATCH(dtype, R, {
    const R inf = R(INFINITY);
    cudaMemcpyAsync(res, &inf, sizeof(R), cudaMemcpyHostToDevice, ctx->stream);
    const R dl = fmin(fmin(R(m->dx), R(m->dy)), R(m->dz));
    cfl_k<R><<<grid_for(ctx, m->n, kThreads, 4), kThreads, 0, ctx->stream>>>(dl, R(gamma), (const R*)p, (const R*)rho,
                                                                              (const R*)u, (const R*)v, (const R*)w, m->n, (R*)res);
    R mn = 0;
    cudaError_t e = cudaMemcpyAsync(&mn, res, sizeof(R), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = cfdb_cuda_fail(ctx, e, "cfdb_cfl_dt");
    host = double(R(cfl) * mn);
  });
  cfdb_ws_free(ctx, res);
  if (rc) return rc;
  if (!std::isfinite(host) || !(host > 0)) return cfdb_fail(ctx, CFDB_ENUMERIC, "cfdb_cfl_dt: non-finite or non-positive dt %g", host);
  *dt_out = host;
  return CFDB_OK;
}

extern "C" int cfdb_total_fp64(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* field, double* out) {
  if (int rc = cfdb_check_mesh(ctx, m)) return rc;
  if (!dtype_ok(dtype)) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_total_fp64: unknown dtype %d", dtype);
  if (int rc = check_ptrs(ctx, "cfdb_total_fp64", {field, out})) return rc;
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  const void* vol = nullptr;
  if (!m->uniform) {
    if (int rc = cfdb_mesh_need_plain(m, dtype)) return rc;
    vol = m->plain[dtype == CFDB_F64 ? 1 : 0].volume;
  }
  const double vconst = m->dx * m->dy * m->dz;
  const int grid = grid_for(ctx, m->n, kThreads, 2);
  void* scratch = nullptr;
  if (int rc = cfdb_ws_alloc(ctx, int64_t(sizeof(Comp)) * grid + 16, &scratch)) return rc;
  Comp* part = static_cast<Comp*>(scratch);
  double* res = reinterpret_cast<double*>(part + grid);
  DISPATCH(dtype, R, total_k<R><<<grid, kThreads, 0, ctx->stream>>>((const R*)field, (const R*)vol, vconst, m->n, part));
  total_final_k<<<1, 32, 0, ctx->stream>>>(part, grid, res);
  cudaError_t e = cudaMemcpyAsync(out, res, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cfdb_ws_free(ctx, scratch);
  if (e != cudaSuccess) return cfdb_cuda_fail(ctx, e, "cfdb_total_fp64");
  return CFDB_OK;
}

int plain_wave_step(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* q, void* qn, const void* c, double cconst,
                    int mode, double dt) {
  if (int rc = cfdb_mesh_need_plain(m, dtype)) return rc;
  DISPATCH(dtype, R, wave_plain_k<R><<<grid_for(ctx, m->n, kThreads), kThreads, 0, ctx->stream>>>(
                         plain_args<R>(m, dtype), (const R*)q, (R*)qn, (const R*)c, R(cconst), mode, R(dt)));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}

int plain_wave_adjoint(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* q, const void* lam1, void* lam0,
                       const void* c, void* gc, double dt) {
  if (int rc = cfdb_mesh_need_plain(m, dtype)) return rc;
  DISPATCH(dtype, R, wave_adjoint_plain_k<R><<<grid_for(ctx, m->n, kThreads), kThreads, 0, ctx->stream>>>(
                         plain_args<R>(m, dtype), (const R*)q, (const R*)lam1, (R*)lam0, (const R*)c, (R*)gc, R(dt)));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}
