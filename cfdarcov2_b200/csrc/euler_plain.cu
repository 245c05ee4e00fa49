// Compressible Euler on the plain (general-geometry) path, float and double,
// plus the reduction kernel both paths use for the per-direction signal
// speeds, the FP64 Neumaier totals and the device clock.  Compiled with
// --fmad=false: the FP64 plain step reproduces the CPU oracle bit for bit.
//
// Scheme (first-order Rusanov, conserved U = [rho|mx|my|mz|E]):
//   F* = (F_P + F_N).n/2 - lam_max (U_N - U_P)/2,  lam_max = max(|u_n| + a)
//   U' = U - dt/V sum_f F* A
// Boundary faces in slots 4/5 (the x ends) are zero-gradient; the others are
// reflective walls (normal momentum negated).
#include <cmath>

#include "euler_internal.hpp"

CFDB_MODULE_ANCHOR

namespace {

constexpr int kThreads = 256;

template <class R> struct Prim { R u, v, w, p, a; };

template <class R> __device__ __forceinline__ Prim<R> prim(R rho, R mx, R my, R mz, R E, R gamma) {
  Prim<R> s;
  s.u = mx / rho; s.v = my / rho; s.w = mz / rho;
  const R ke = R(0.5) * ((mx * s.u + my * s.v) + mz * s.w);
  s.p = (gamma - R(1)) * (E - ke);
  s.a = sqrt(gamma * s.p / rho);
  return s;
}

__device__ __forceinline__ double bits_to_double(unsigned long long b) { return __longlong_as_double((long long)b); }

template <class R> struct PlainEulerArgs {
  const int32_t* __restrict__ ids;
  const R* __restrict__ nalt;  // 3 x 6n
  const R* __restrict__ area;
  const R* __restrict__ vol;
  long long n;
  R gamma;
  double dx, dy, dz, cfl, t_end;
  EulerClock* clock;
};

template <class R>
__global__ void __launch_bounds__(kThreads) euler_plain_step_k(PlainEulerArgs<R> g, const R* __restrict__ U,
                                                               R* __restrict__ Un, long long s) {
  const EulerClock* ck = g.clock;
  const int ts = int(s & 1);
  if (ck->finished[ts]) return;
  const int ls = int(s % 3);
  const double lam[3] = {bits_to_double(ck->lam[ls][0]), bits_to_double(ck->lam[ls][1]), bits_to_double(ck->lam[ls][2])};
  bool last;
  const R dt = R(euler_dt(lam, g.dx, g.dy, g.dz, g.cfl, ck->t[ts], g.t_end, &last));
  const long long n = g.n;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const R rP = U[i], mxP = U[n + i], myP = U[2 * n + i], mzP = U[3 * n + i], EP = U[4 * n + i];
    const Prim<R> P = prim(rP, mxP, myP, mzP, EP, g.gamma);
    R acc[5] = {R(0), R(0), R(0), R(0), R(0)};
#pragma unroll 1
    for (int f = 0; f < 6; ++f) {
      const long long k6 = (long long)f * n + i;
      const R nx = g.nalt[k6], ny = g.nalt[6 * n + k6], nz = g.nalt[12 * n + k6];
      const R A = g.area[k6];
      const long long j = g.ids[k6];
      R rN, mxN, myN, mzN, EN;
      if (j != i) {
        rN = U[j]; mxN = U[n + j]; myN = U[2 * n + j]; mzN = U[3 * n + j]; EN = U[4 * n + j];
      } else if (f >= 4) {
        rN = rP; mxN = mxP; myN = myP; mzN = mzP; EN = EP;
      } else {
        const R two_mn = R(2) * ((mxP * nx + myP * ny) + mzP * nz);
        rN = rP; mxN = mxP - two_mn * nx; myN = myP - two_mn * ny; mzN = mzP - two_mn * nz; EN = EP;
      }
      const Prim<R> N = prim(rN, mxN, myN, mzN, EN, g.gamma);
      const R unP = (P.u * nx + P.v * ny) + P.w * nz;
      const R unN = (N.u * nx + N.v * ny) + N.w * nz;
      const R lm = fmax(fabs(unP) + P.a, fabs(unN) + N.a);
      const R hl = R(0.5) * lm;
      const R f0 = R(0.5) * (rP * unP + rN * unN) - hl * (rN - rP);
      const R f1 = R(0.5) * ((mxP * unP + P.p * nx) + (mxN * unN + N.p * nx)) - hl * (mxN - mxP);
      const R f2 = R(0.5) * ((myP * unP + P.p * ny) + (myN * unN + N.p * ny)) - hl * (myN - myP);
      const R f3 = R(0.5) * ((mzP * unP + P.p * nz) + (mzN * unN + N.p * nz)) - hl * (mzN - mzP);
      const R f4 = R(0.5) * ((EP + P.p) * unP + (EN + N.p) * unN) - hl * (EN - EP);
      acc[0] = acc[0] + f0 * A; acc[1] = acc[1] + f1 * A; acc[2] = acc[2] + f2 * A;
      acc[3] = acc[3] + f3 * A; acc[4] = acc[4] + f4 * A;
    }
    const R V = g.vol[i];
#pragma unroll
    for (int c = 0; c < 5; ++c) Un[c * n + i] = dt * (-(acc[c] / V)) + U[c * n + i];
  }
}

__device__ __forceinline__ void comp_add(double& s, double& c, double x) {
  const double t = s + x;
  if (fabs(s) >= fabs(x)) c += (s - t) + x; else c += (x - t) + s;
  s = t;
}

// Per-direction max speeds + Neumaier totals of U; the last CTA finalises.
// begin_mode: initial state (ring slot 0, totals row 0, no clock advance).
template <class R>
__global__ void __launch_bounds__(kThreads) euler_reduce_k(const R* __restrict__ U, const R* __restrict__ vol,
                                                           double vconst, long long n, R gamma, double dx, double dy,
                                                           double dz, double cfl, double t_end, EulerClock* ck,
                                                           double* __restrict__ totals, Comp2* __restrict__ part,
                                                           long long s, int begin_mode, long long max_steps) {
  const int ts = int(s & 1);
  if (!begin_mode && ck->finished[ts]) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      ck->t[ts ^ 1] = ck->t[ts];
      ck->steps[ts ^ 1] = ck->steps[ts];
      ck->finished[ts ^ 1] = 1;
    }
    return;
  }
  const int target = begin_mode ? 0 : int((s + 1) % 3);
  if (!begin_mode && blockIdx.x == 0 && threadIdx.x == 0) {
    const int z = int((s + 2) % 3);
    ck->lam[z][0] = ck->lam[z][1] = ck->lam[z][2] = 0ull;
  }
  R lx = R(0), ly = R(0), lz = R(0);
  double s0 = 0, c0 = 0, s1 = 0, c1 = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const R rho = U[i];
    const Prim<R> P = prim(rho, U[n + i], U[2 * n + i], U[3 * n + i], U[4 * n + i], gamma);
    lx = fmax(lx, fabs(P.u) + P.a);
    ly = fmax(ly, fabs(P.v) + P.a);
    lz = fmax(lz, fabs(P.w) + P.a);
    const double V = vol ? double(vol[i]) : vconst;
    comp_add(s0, c0, double(rho) * V);
    comp_add(s1, c1, double(U[4 * n + i]) * V);
  }
  // block reduction (fixed tree: deterministic for a fixed grid)
  __shared__ double sh[kThreads / 32][4];
  __shared__ R shl[kThreads / 32][3];
  __shared__ bool is_last;
  for (int o = 16; o > 0; o >>= 1) {
    lx = fmax(lx, __shfl_xor_sync(0xffffffffu, lx, o));
    ly = fmax(ly, __shfl_xor_sync(0xffffffffu, ly, o));
    lz = fmax(lz, __shfl_xor_sync(0xffffffffu, lz, o));
    const double a0 = __shfl_xor_sync(0xffffffffu, s0, o), b0 = __shfl_xor_sync(0xffffffffu, c0, o);
    const double a1 = __shfl_xor_sync(0xffffffffu, s1, o), b1 = __shfl_xor_sync(0xffffffffu, c1, o);
    comp_add(s0, c0, a0); c0 += b0;
    comp_add(s1, c1, a1); c1 += b1;
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    sh[w][0] = s0; sh[w][1] = c0; sh[w][2] = s1; sh[w][3] = c1;
    shl[w][0] = lx; shl[w][1] = ly; shl[w][2] = lz;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double S0 = 0, C0 = 0, S1 = 0, C1 = 0;
    R L0 = 0, L1 = 0, L2 = 0;
    for (int k = 0; k < kThreads / 32; ++k) {
      comp_add(S0, C0, sh[k][0]); C0 += sh[k][1];
      comp_add(S1, C1, sh[k][2]); C1 += sh[k][3];
      L0 = fmax(L0, shl[k][0]); L1 = fmax(L1, shl[k][1]); L2 = fmax(L2, shl[k][2]);
    }
    part[blockIdx.x] = Comp2{S0, C0, S1, C1};
    atomicMax(&ck->lam[target][0], (unsigned long long)__double_as_longlong(double(L0)));
    atomicMax(&ck->lam[target][1], (unsigned long long)__double_as_longlong(double(L1)));
    atomicMax(&ck->lam[target][2], (unsigned long long)__double_as_longlong(double(L2)));
    __threadfence();
    is_last = atomicAdd(&ck->counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (is_last && threadIdx.x == 0) {
    __threadfence();
    double S0 = 0, C0 = 0, S1 = 0, C1 = 0;
    for (unsigned k = 0; k < gridDim.x; ++k) {
      const Comp2 p = part[k];
      comp_add(S0, C0, p.s0); C0 += p.c0;
      comp_add(S1, C1, p.s1); C1 += p.c1;
    }
    ck->counter = 0;
    if (begin_mode) {
      totals[0] = S0 + C0;
      totals[1] = S1 + C1;
    } else {
      const int ls = int(s % 3);
      const double lam[3] = {bits_to_double(ck->lam[ls][0]), bits_to_double(ck->lam[ls][1]), bits_to_double(ck->lam[ls][2])};
      bool last;
      const double t = ck->t[ts];
      const double dt = euler_dt(lam, dx, dy, dz, cfl, t, t_end, &last);
      const long long step = ck->steps[ts] + 1;
      ck->t[ts ^ 1] = last ? t_end : t + dt;
      ck->steps[ts ^ 1] = step;
      ck->finished[ts ^ 1] = (last || !(t + dt < t_end) || step >= max_steps) ? 1 : 0;
      totals[2 * step] = S0 + C0;
      totals[2 * step + 1] = S1 + C1;
    }
  }
}

}  // namespace

int euler_reduce_grid(const cfdb_euler* e) { return grid_for(e->ctx, e->mesh->n, kThreads, 2); }

int euler_plain_step(cfdb_euler* e, const void* U, void* Un, int64_t s) {
  cfdb_ctx* ctx = e->ctx;
  cfdb_mesh* m = e->mesh;
  if (int rc = cfdb_mesh_need_plain(m, e->dtype)) return rc;
  const PlainGeomDev& p = m->plain[e->dtype == CFDB_F64 ? 1 : 0];
  const int grid = grid_for(ctx, m->n, kThreads, 8);
  if (e->dtype == CFDB_F64) {
    PlainEulerArgs<double> a{m->d_ids, (const double*)p.normal_alt, (const double*)p.area, (const double*)p.volume,
                             (long long)m->n, e->gamma, m->dx, m->dy, m->dz, e->cfl, e->t_end, e->clock};
    euler_plain_step_k<double><<<grid, kThreads, 0, ctx->stream>>>(a, (const double*)U, (double*)Un, s);
  } else {
    PlainEulerArgs<float> a{m->d_ids, (const float*)p.normal_alt, (const float*)p.area, (const float*)p.volume,
                            (long long)m->n, float(e->gamma), m->dx, m->dy, m->dz, e->cfl, e->t_end, e->clock};
    euler_plain_step_k<float><<<grid, kThreads, 0, ctx->stream>>>(a, (const float*)U, (float*)Un, s);
  }
  CFDB_LAUNCHED(ctx);
  return euler_reduce(e, Un, s, 0);
}

int euler_reduce(cfdb_euler* e, const void* U, int64_t s, int begin_mode) {
  cfdb_ctx* ctx = e->ctx;
  cfdb_mesh* m = e->mesh;
  const void* vol = nullptr;
  if (e->path == CFDB_PATH_PLAIN || !m->uniform) {
    if (int rc = cfdb_mesh_need_plain(m, e->dtype)) return rc;
    vol = m->plain[e->dtype == CFDB_F64 ? 1 : 0].volume;
  }
  const double vconst = m->dx * m->dy * m->dz;
  const int grid = euler_reduce_grid(e);
  if (e->dtype == CFDB_F64)
    euler_reduce_k<double><<<grid, kThreads, 0, ctx->stream>>>((const double*)U, (const double*)vol, vconst, (long long)m->n,
                                                                e->gamma, m->dx, m->dy, m->dz, e->cfl, e->t_end, e->clock,
                                                                e->totals, e->part, s, begin_mode, (long long)e->max_steps);
  else
    euler_reduce_k<float><<<grid, kThreads, 0, ctx->stream>>>((const float*)U, (const float*)vol, vconst, (long long)m->n,
                                                               float(e->gamma), m->dx, m->dy, m->dz, e->cfl, e->t_end,
                                                               e->clock, e->totals, e->part, s, begin_mode,
                                                               (long long)e->max_steps);
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}
