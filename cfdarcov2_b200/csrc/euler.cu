// Compressible Euler solver object (cfdb_euler_*) and its fused FP32 step:
// one face-flux TMA sweep per step (face_sweep.cuh) that reads the device clock, does
// the Rusanov update of all five conserved fields in one HBM pass and, in its
// epilogue, reduces the new state's per-direction signal speeds (for the next
// dt) and its FP64 Neumaier totals.  The plain path lives in euler_plain.cu.
#include <cmath>
#include <new>

#include "euler_internal.hpp"
#include "f32x2.cuh"
#include "tma_host.hpp"

CFDB_MODULE_ANCHOR

namespace {

__device__ __forceinline__ double bits_to_double(unsigned long long b) { return __longlong_as_double((long long)b); }

__device__ __forceinline__ void comp_add(double& s, double& c, double x) {
  const double t = s + x;
  if (fabs(s) >= fabs(x)) c += (s - t) + x; else c += (x - t) + s;
  s = t;
}

// Folds the per-CTA FP64 partials part[0 .. nblocks) into totals row `step`
// with every thread of the calling CTA, in a fixed order: thread t takes
// partials t, t + blockDim, ..., the lanes of each warp merge through
// shuffles in a fixed pattern and thread 0 merges the warps in order, so the
// totals do not depend on timing (one thread folding every partial serially
// had cost ~13 us per step).
__device__ void fold_partials(const Comp2* __restrict__ part, int nblocks, double* totals, long long step) {
  __shared__ double sh[32][4];
  double S0 = 0, C0 = 0, S1 = 0, C1 = 0;
  for (int k = int(threadIdx.x); k < nblocks; k += int(blockDim.x)) {
    const Comp2 q = part[k];
    comp_add(S0, C0, q.s0); C0 += q.c0;
    comp_add(S1, C1, q.s1); C1 += q.c1;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double a0 = __shfl_xor_sync(0xffffffffu, S0, o), b0 = __shfl_xor_sync(0xffffffffu, C0, o);
    const double a1 = __shfl_xor_sync(0xffffffffu, S1, o), b1 = __shfl_xor_sync(0xffffffffu, C1, o);
    comp_add(S0, C0, a0); C0 += b0;
    comp_add(S1, C1, a1); C1 += b1;
  }
  const int w = int(threadIdx.x) >> 5;
  if ((threadIdx.x & 31) == 0) {
    sh[w][0] = S0; sh[w][1] = C0; sh[w][2] = S1; sh[w][3] = C1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    S0 = C0 = S1 = C1 = 0;
    for (int k = 0; k < int(blockDim.x / 32); ++k) {
      comp_add(S0, C0, sh[k][0]); C0 += sh[k][1];
      comp_add(S1, C1, sh[k][2]); C1 += sh[k][3];
    }
    totals[2 * step] = S0 + C0;
    totals[2 * step + 1] = S1 + C1;
  }
}

struct EulerPhys {
  static constexpr int NF = 5;
  static constexpr int MIN_BLOCKS = 2;  // 64x8 tile, 2 cells per thread: 256 threads at <= 128 registers
  struct Params {
    float ih[3];
    float gamma;
    float dt;     // filled per launch by begin()
    float kd[3];  // dt / h_d, filled per launch by begin()
    double dx, dy, dz, cfl, t_end, vconst;
    EulerClock* clock;
    double* totals;
    Comp2* part;      // two buffers of part_stride partials, launch s writes buffer s % 2
    int part_stride;
    long long s;
    long long max_steps;
  };
  struct Acc {
    float l[3];
    double s0, c0, s1, c1;
  };

  __device__ static bool first_thread() {
    return blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0;
  }

  // The clock of the new state is written when the step starts (it needs
  // only dt); the totals of the previous launch's state are folded by this
  // launch's first CTA while its first planes are in flight (prologue), or
  // here when nothing is left to step.
  __device__ static bool begin(Params& p) {
    EulerClock* ck = p.clock;
    const int ts = int(p.s & 1);
    if (ck->finished[ts]) {
      fold_previous(p);
      if (first_thread()) {
        ck->t[ts ^ 1] = ck->t[ts];
        ck->steps[ts ^ 1] = ck->steps[ts];
        ck->finished[ts ^ 1] = 1;
        ck->pending[ts] = 0;
      }
      return false;
    }
    if (first_thread()) {
      const int z = int((p.s + 2) % 3);
      ck->lam[z][0] = ck->lam[z][1] = ck->lam[z][2] = 0ull;
    }
    const int ls = int(p.s % 3);
    const double lam[3] = {bits_to_double(ck->lam[ls][0]), bits_to_double(ck->lam[ls][1]),
                           bits_to_double(ck->lam[ls][2])};
    bool last;
    const double t = ck->t[ts];
    const double dt = euler_dt(lam, p.dx, p.dy, p.dz, p.cfl, t, p.t_end, &last);
    p.dt = float(dt);
    for (int d = 0; d < 3; ++d) p.kd[d] = p.dt * p.ih[d];
    if (first_thread()) {
      const long long step = ck->steps[ts] + 1;
      ck->t[ts ^ 1] = last ? p.t_end : t + dt;
      ck->steps[ts ^ 1] = step;
      ck->finished[ts ^ 1] = (last || !(t + dt < p.t_end) || step >= p.max_steps) ? 1 : 0;
      ck->pending[ts] = step;
    }
    return true;
  }
  // The first CTA folds the partials the previous launch left (if it
  // stepped) into that step's totals row.
  __device__ static void fold_previous(const Params& p) {
    if (blockIdx.x != 0 || blockIdx.y != 0 || p.s < 1) return;
    const int prev = int((p.s - 1) & 1);
    const long long step = p.clock->pending[prev];
    if (step <= 0) return;
    fold_partials(p.part + size_t(prev) * size_t(p.part_stride), int(gridDim.x * gridDim.y), p.totals, step);
  }
  __device__ static void prologue(const Params& p) { fold_previous(p); }


  // 1/rho and the sound speed with the approximate reciprocal and square
  // root of the SFU (relative error ~1e-7, far inside the FP32 solver's
  // 1e-5 error bar against FP64; the FP64 path keeps IEEE division).
  __device__ static float fast_rcp(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
  }
  __device__ static float fast_sqrt(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
  }

  __device__ static void prim(const float q[NF], float gm1, float gamma, float& ir, float u[3], float& p, float& a) {
    ir = fast_rcp(q[0]);
    u[0] = q[1] * ir; u[1] = q[2] * ir; u[2] = q[3] * ir;
    p = gm1 * (q[4] - 0.5f * (q[1] * u[0] + q[2] * u[1] + q[3] * u[2]));
    a = fast_sqrt(gamma * p * ir);
  }

  // Derived per cell, computed once per cell and plane by the sweep:
  // d = (1/rho, p, a).  A reflective or zero-gradient ghost has the same
  // values as its cell (ghost() copies them).
  static constexpr int ND = 3;
  static constexpr int NG = 0;   // uniform mesh: no per-cell geometry
  static constexpr int NGF = 0;
  __device__ static void derive(const float q[NF], float d[ND], const Params& a) {
    float u[3];
    prim(q, a.gamma - 1.0f, a.gamma, d[0], u, d[1], d[2]);
  }

  // Rusanov flux through a face with normal +e_d, L on its minus side:
  //   F = (F_L + F_R)/2 . e_d - lambda/2 (U_R - U_L),  lambda = max(|u_d| + a)
  // regrouped per conserved component U as U_L (u_L/2 + l) + U_R (u_R/2 - l)
  // with l = lambda/2 (two instructions per component), the pressure terms
  // added to the momentum and energy components.  The sweep evaluates each
  // face once and enters it into the two cells it separates with opposite
  // signs.
  __device__ static void flux(const float L[NF], const float Ld[ND], const float R[NF], const float Rd[ND],
                              const float*, int d, const Params&, float F[NF]) {
    const float uL = L[1 + d] * Ld[0], uR = R[1 + d] * Rd[0];
    const float pL = Ld[1], pR = Rd[1];
    const float l = 0.5f * fmaxf(fabsf(uL) + Ld[2], fabsf(uR) + Rd[2]);
    const float wL = 0.5f * uL + l, wR = 0.5f * uR - l;
#pragma unroll
    for (int c = 0; c < NF; ++c) F[c] = L[c] * wL + R[c] * wR;
    F[1 + d] += 0.5f * (pL + pR);
    F[4] += 0.5f * (pL * uL + pR * uR);
  }
  // Walls: a face on the domain boundary is evaluated against a ghost cell,
  // which the sweep builds for every face that can be a wall and selects
  // (SELECT_WALLS: a few selects, no branch around the flux).  Zero-gradient
  // at the x ends (a copy), reflective in y and z (the wall-normal momentum
  // negated); 1/rho, p and a are the cell's own.
  static constexpr bool SELECT_WALLS = true;
  __device__ static void ghost(const float C[NF], const float Cd[ND], const float*, int d, float g[NF], float gd[ND]) {
#pragma unroll
    for (int f = 0; f < NF; ++f) g[f] = C[f];
    if (d == 1) g[2] = -C[2];
    if (d == 2) g[3] = -C[3];
#pragma unroll
    for (int e = 0; e < ND; ++e) gd[e] = Cd[e];
  }
  __device__ static void acc_init(Acc& s) {
    s.l[0] = s.l[1] = s.l[2] = 0.f;
    s.s0 = s.c0 = s.s1 = s.c1 = 0.0;
  }

  // The sweep runs two z cells per thread and hands them over as (cell 0,
  // cell 1) pairs: every FP32 add, multiply and fma below is one packed
  // f32x2 instruction (each lane rounds like the scalar instruction); the
  // reciprocal, square root, |.| and max stay per lane.  The scalar flux
  // and derive above serve the single faces and halo cells.
  static constexpr bool PAIRED = true;
  __device__ static float2 rcp2(float2 x) { return make_float2(fast_rcp(x.x), fast_rcp(x.y)); }
  __device__ static float2 sqrt2(float2 x) { return make_float2(fast_sqrt(x.x), fast_sqrt(x.y)); }
  __device__ static void prim2(const float2 q[NF], const Params& a, float2& ir, float2 u[3], float2& p, float2& c) {
    using namespace f2;
    ir = rcp2(q[0]);
    u[0] = mul(q[1], ir); u[1] = mul(q[2], ir); u[2] = mul(q[3], ir);
    const float2 ke = fma(q[3], u[2], fma(q[2], u[1], mul(q[1], u[0])));
    p = mul(splat(a.gamma - 1.0f), fma(splat(-0.5f), ke, q[4]));
    c = sqrt2(mul(mul(splat(a.gamma), p), ir));
  }
  __device__ static void derive2(const float2 q[NF], float2 d[ND], const Params& a) {
    float2 u[3];
    prim2(q, a, d[0], u, d[1], d[2]);
  }
  __device__ static void flux2(const float2 L[NF], const float2 Ld[ND], const float2 R[NF], const float2 Rd[ND], int d,
                               const Params&, float2 F[NF]) {
    using namespace f2;
    const float2 uL = mul(L[1 + d], Ld[0]), uR = mul(R[1 + d], Rd[0]);
    const float2 pL = Ld[1], pR = Rd[1];
    const float2 m = make_float2(fmaxf(fabsf(uL.x) + Ld[2].x, fabsf(uR.x) + Rd[2].x),
                                 fmaxf(fabsf(uL.y) + Ld[2].y, fabsf(uR.y) + Rd[2].y));
    const float2 h = splat(0.5f);
    const float2 wL = fma(h, uL, mul(h, m)), wR = fma(h, uR, mul(splat(-0.5f), m));
#pragma unroll
    for (int c = 0; c < NF; ++c) F[c] = fma(L[c], wL, mul(R[c], wR));
    F[1 + d] = fma(h, add(pL, pR), F[1 + d]);
    F[4] = fma(h, fma(pL, uL, mul(pR, uR)), F[4]);
  }
  // Update: U' = U - sum_d (dt/h_d) (F(d+) - F(d-)).
  __device__ static void update2(const float2 P[NF], const float2*, const float2 dF[3][NF], const Params& a,
                                 float2 o[NF]) {
    using namespace f2;
    const float2 k0 = splat(a.kd[0]), k1 = splat(a.kd[1]), k2 = splat(a.kd[2]);
#pragma unroll
    for (int c = 0; c < NF; ++c) o[c] = sub(P[c], fma(k0, dF[0][c], fma(k1, dF[1][c], mul(k2, dF[2][c]))));
  }
  // Epilogue per cell of the new state: the signal speeds |u_d| + a for the
  // next dt, and the mass and energy summed in plain double (with 24-bit
  // inputs the error of a thread's few hundred cells stays near 1e-13
  // relative; compensation starts where the per-thread sums meet).  The
  // uniform volume multiplies once.
  __device__ static void acc_cell2(Acc& s, const float2 o[NF], const Params& a) {
    float2 ir, u[3], p, c;
    prim2(o, a, ir, u, p, c);
#pragma unroll
    for (int i = 0; i < 3; ++i) s.l[i] = fmaxf(s.l[i], fmaxf(fabsf(u[i].x) + c.x, fabsf(u[i].y) + c.y));
    s.s0 += double(o[0].x) + double(o[0].y);
    s.s1 += double(o[4].x) + double(o[4].y);
  }

  __device__ static void finish(Acc& s, const Params& a, bool) {
    __shared__ double sh[32][4];
    __shared__ float shl[32][3];
    s.s0 *= a.vconst;
    s.s1 *= a.vconst;
    for (int o = 16; o > 0; o >>= 1) {
      s.l[0] = fmaxf(s.l[0], __shfl_xor_sync(0xffffffffu, s.l[0], o));
      s.l[1] = fmaxf(s.l[1], __shfl_xor_sync(0xffffffffu, s.l[1], o));
      s.l[2] = fmaxf(s.l[2], __shfl_xor_sync(0xffffffffu, s.l[2], o));
      const double a0 = __shfl_xor_sync(0xffffffffu, s.s0, o), b0 = __shfl_xor_sync(0xffffffffu, s.c0, o);
      const double a1 = __shfl_xor_sync(0xffffffffu, s.s1, o), b1 = __shfl_xor_sync(0xffffffffu, s.c1, o);
      comp_add(s.s0, s.c0, a0); s.c0 += b0;
      comp_add(s.s1, s.c1, a1); s.c1 += b1;
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
      sh[w][0] = s.s0; sh[w][1] = s.c0; sh[w][2] = s.s1; sh[w][3] = s.c1;
      shl[w][0] = s.l[0]; shl[w][1] = s.l[1]; shl[w][2] = s.l[2];
    }
    __syncthreads();
    EulerClock* ck = a.clock;
    const unsigned bid = blockIdx.y * gridDim.x + blockIdx.x;
    if (threadIdx.x == 0) {
      double S0 = 0, C0 = 0, S1 = 0, C1 = 0;
      float L0 = 0, L1 = 0, L2 = 0;
      for (int k = 0; k < int(blockDim.x / 32); ++k) {
        comp_add(S0, C0, sh[k][0]); C0 += sh[k][1];
        comp_add(S1, C1, sh[k][2]); C1 += sh[k][3];
        L0 = fmaxf(L0, shl[k][0]); L1 = fmaxf(L1, shl[k][1]); L2 = fmaxf(L2, shl[k][2]);
      }
      a.part[size_t(a.s & 1) * size_t(a.part_stride) + bid] = Comp2{S0, C0, S1, C1};
      const int target = int((a.s + 1) % 3);
      atomicMax(&ck->lam[target][0], (unsigned long long)__double_as_longlong(double(L0)));
      atomicMax(&ck->lam[target][1], (unsigned long long)__double_as_longlong(double(L1)));
      atomicMax(&ck->lam[target][2], (unsigned long long)__double_as_longlong(double(L2)));
    }
  }
};

// The fold of the partials the last launch left, for a reader of the totals
// after the last step (cfdb_euler_totals, the run loop's health check).
__global__ void euler_fold_k(EulerClock* ck, const Comp2* __restrict__ part, int stride, int nblocks,
                             double* totals, int prev) {
  const long long step = ck->pending[prev];
  if (step <= 0) return;
  fold_partials(part + size_t(prev) * size_t(stride), nblocks, totals, step);
}

constexpr int kEulerCtasPerSm = 2;
constexpr int kEulerVZ = 2;

static_assert(kEulerVZ == 2, "EulerPhys provides its per-cell update only as packed pairs");

template <int TZ>
int launch_euler(cfdb_euler* e, const void* U, void* Un, int64_t s) {
  cfdb_mesh* m = e->mesh;
  EulerPhys::Params p;
  p.ih[0] = float(1.0 / m->dx); p.ih[1] = float(1.0 / m->dy); p.ih[2] = float(1.0 / m->dz);
  p.gamma = float(e->gamma);
  p.dt = 0.f;
  p.dx = m->dx; p.dy = m->dy; p.dz = m->dz;
  p.cfl = e->cfl; p.t_end = e->t_end; p.vconst = m->dx * m->dy * m->dz;
  p.clock = e->clock; p.totals = e->totals; p.part = e->part;
  p.s = (long long)s;
  p.max_steps = (long long)e->max_steps;
  p.part_stride = e->part_cap;
  const stencil::PaddedGeom none{nullptr, 0, 0, 0, 0};
  int grid = 0;
  const int rc =
      stencil::launch_face_sweep<EulerPhys, TZ, 8, 4, kEulerVZ>(e->ctx, m, U, none, Un, p, kEulerCtasPerSm, &grid);
  if (rc) return rc;
  if (grid > e->part_cap) return cfdb_fail(e->ctx, CFDB_ECUDA, "fused Euler grid %d beyond its %d partials", grid, e->part_cap);
  e->fused_grid = grid;
  e->fused_threads = (TZ / kEulerVZ) * 8;
  return CFDB_OK;
}

int tz_for(const cfdb_mesh* m) { return m->nz >= 64 ? 64 : 32; }

}  // namespace

// Upper bound of the fused Euler grid (sizes the per-CTA partials): at most
// kEulerCtasPerSm resident CTAs per SM are ever requested.
int euler_fused_grid(const cfdb_euler* e) {
  const int tz = tz_for(e->mesh);
  const stencil::SweepShape sh = stencil::sweep_shape(e->ctx, e->mesh, tz, 8, kEulerCtasPerSm);
  return sh.tiles * sh.chunks;
}

// Folds the partials the last fused launch left into its totals row (a
// no-op when that launch already had its totals folded by a later one, or
// did not step).
int euler_fold_pending(cfdb_euler* e) {
  if (e->path != CFDB_PATH_FUSED || e->launches < 1 || e->fused_grid < 1) return CFDB_OK;
  const int prev = int((e->launches - 1) & 1);
  euler_fold_k<<<1, e->fused_threads, 0, e->ctx->stream>>>(e->clock, e->part, e->part_cap, e->fused_grid, e->totals,
                                                          prev);
  CFDB_LAUNCHED(e->ctx);
  return CFDB_OK;
}

int euler_fused_step(cfdb_euler* e, const void* U, void* Un, int64_t s) {
  switch (tz_for(e->mesh)) {
    case 64: return launch_euler<64>(e, U, Un, s);
    default: return launch_euler<32>(e, U, Un, s);
  }
}

// ---------------------------------------------------------------------------
// object API
// ---------------------------------------------------------------------------
extern "C" int cfdb_euler_create(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, int path, double gamma, double cfl,
                                 double t_end, int64_t max_steps, cfdb_euler** out) {
  if (!out) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_euler_create: out is NULL");
  *out = nullptr;
  if (int rc = cfdb_check_mesh(ctx, m)) return rc;
  if (!dtype_ok(dtype)) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_euler_create: unknown dtype %d", dtype);
  if (path != CFDB_PATH_PLAIN && path != CFDB_PATH_FUSED)
    return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_euler_create: unknown path %d", path);
  if (!(gamma > 1.0) || !(cfl > 0.0) || !(t_end > 0.0) || !std::isfinite(t_end) || max_steps < 1)
    return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_euler_create: need gamma > 1, cfl > 0, finite t_end > 0, max_steps >= 1");
  if (path == CFDB_PATH_FUSED) {
    if (dtype != CFDB_F32) return cfdb_fail(ctx, CFDB_EUNSUPPORTED, "the fused Euler step computes in float32 only");
    if (int rc = stencil::check_sweep(ctx, m, {})) return rc;
  }
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  auto* e = new (std::nothrow) cfdb_euler();
  if (!e) return cfdb_fail(ctx, CFDB_ENOMEM, "host allocation failed");
  e->ctx = ctx; e->mesh = m; e->dtype = dtype; e->path = path;
  e->gamma = gamma; e->cfl = cfl; e->t_end = t_end; e->max_steps = max_steps;
  const int grid = std::max(euler_reduce_grid(e), path == CFDB_PATH_FUSED ? euler_fused_grid(e) : 0);
  e->part_cap = grid;
  int rc = cfdb_dev_alloc(ctx, sizeof(EulerClock), reinterpret_cast<void**>(&e->clock));
  if (!rc) rc = cfdb_dev_alloc(ctx, int64_t(sizeof(double)) * 2 * (max_steps + 1), reinterpret_cast<void**>(&e->totals));
  if (!rc) rc = cfdb_dev_alloc(ctx, int64_t(sizeof(Comp2)) * grid * 2, reinterpret_cast<void**>(&e->part));
  if (rc) {
    cfdb_euler_destroy(e);
    return rc;
  }
  cudaMemsetAsync(e->clock, 0, sizeof(EulerClock), ctx->stream);
  cfdb_adopt(ctx, e, [e] { e->ctx = nullptr; e->clock = nullptr; e->totals = nullptr; e->part = nullptr; });
  *out = e;
  return CFDB_OK;
}

extern "C" int cfdb_euler_destroy(cfdb_euler* e) {
  if (!e) return CFDB_OK;
  if (e->ctx) {
    cfdb_release(e->ctx, e);
    cudaStreamSynchronize(e->ctx->stream);
    cfdb_dev_free(e->ctx, e->clock);
    cfdb_dev_free(e->ctx, e->totals);
    cfdb_dev_free(e->ctx, e->part);
  }
  delete e;
  return CFDB_OK;
}

extern "C" int cfdb_euler_begin(cfdb_euler* e, const void* U0) {
  if (!e || !e->ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_euler_begin: handle is NULL or its context was destroyed");
  if (!U0) return cfdb_fail(e->ctx, CFDB_EINVAL, "cfdb_euler_begin: U0 is NULL");
  if (e->path == CFDB_PATH_FUSED && (reinterpret_cast<uintptr_t>(U0) & 15u))
    return cfdb_fail(e->ctx, CFDB_EINVAL, "the fused Euler path needs 16-byte aligned states");
  CFDB_CUDA(e->ctx, cudaSetDevice(e->ctx->device));
  CFDB_CUDA(e->ctx, cudaMemsetAsync(e->clock, 0, sizeof(EulerClock), e->ctx->stream));
  e->launches = 0;
  return euler_reduce(e, U0, 0, 1);
}

extern "C" int cfdb_euler_step(cfdb_euler* e, const void* U, void* Un) {
  if (!e || !e->ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_euler_step: handle is NULL or its context was destroyed");
  if (!U || !Un || U == Un) return cfdb_fail(e->ctx, CFDB_EINVAL, "cfdb_euler_step: need distinct U and U_next");
  CFDB_CUDA(e->ctx, cudaSetDevice(e->ctx->device));
  const int64_t s = e->launches;
  int rc = e->path == CFDB_PATH_FUSED ? euler_fused_step(e, U, Un, s) : euler_plain_step(e, U, Un, s);
  if (rc) return rc;
  e->launches = s + 1;
  return CFDB_OK;
}

extern "C" int cfdb_euler_status(cfdb_euler* e, double* t, int64_t* steps_done, int* finished) {
  if (!e || !e->ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_euler_status: handle is NULL or its context was destroyed");
  EulerClock ck;
  CFDB_CUDA(e->ctx, cudaMemcpyAsync(&ck, e->clock, sizeof(ck), cudaMemcpyDeviceToHost, e->ctx->stream));
  CFDB_CUDA(e->ctx, cudaStreamSynchronize(e->ctx->stream));
  if (int rc = cfdb_check_device_error(e->ctx)) return rc;
  const int sl = euler_slot(e->launches);
  if (t) *t = ck.t[sl];
  if (steps_done) *steps_done = ck.steps[sl];
  if (finished) *finished = ck.finished[sl];
  return CFDB_OK;
}

extern "C" int cfdb_euler_totals(cfdb_euler* e, double* out, int64_t max_rows, int64_t* rows) {
  if (!e || !e->ctx || !out || max_rows < 0)
    return cfdb_fail(e ? e->ctx : nullptr, CFDB_EINVAL, "cfdb_euler_totals: bad arguments");
  int64_t steps = 0;
  if (int rc = euler_fold_pending(e)) return rc;
  if (int rc = cfdb_euler_status(e, nullptr, &steps, nullptr)) return rc;
  const int64_t n = std::min<int64_t>(steps + 1, max_rows);
  if (n > 0) CFDB_CUDA(e->ctx, cudaMemcpy(out, e->totals, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost));
  if (rows) *rows = n;
  return CFDB_OK;
}

extern "C" int cfdb_euler_run(cfdb_euler* e, void* Ua, void* Ub, int64_t check_every, int64_t* steps_done,
                              int* final_in_b) {
  CfdbRange range_("cfdb_euler_run");
  if (!e || !e->ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_euler_run: handle is NULL or its context was destroyed");
  if (!Ua || !Ub || Ua == Ub || check_every < 1)
    return cfdb_fail(e->ctx, CFDB_EINVAL, "cfdb_euler_run: need distinct buffers and check_every >= 1");
  if (e->launches & 1) return cfdb_fail(e->ctx, CFDB_EINVAL, "cfdb_euler_run: call after cfdb_euler_begin or an even number of steps");
  int finished = 0;
  int64_t steps = 0;
  while (!finished) {
    for (int64_t k = 0; k < check_every; ++k) {
      const bool even = (e->launches & 1) == 0;
      if (int rc = cfdb_euler_step(e, even ? Ua : Ub, even ? Ub : Ua)) return rc;
    }
    if (int rc = euler_fold_pending(e)) return rc;
    if (int rc = cfdb_euler_status(e, nullptr, &steps, &finished)) return rc;
    // the conservation totals of the latest step double as the health check:
    // a NaN or Inf anywhere in the state reaches them (and would otherwise
    // end the run early through a non-finite dt)
    double last[2] = {0.0, 0.0};
    CFDB_CUDA(e->ctx, cudaMemcpy(last, e->totals + 2 * steps, sizeof(last), cudaMemcpyDeviceToHost));
    if (!std::isfinite(last[0]) || !std::isfinite(last[1]))
      return cfdb_fail(e->ctx, CFDB_ENUMERIC, "cfdb_euler_run: the state is not finite at step %lld (totals %g, %g)",
                       (long long)steps, last[0], last[1]);
    if (!finished && e->launches > e->max_steps + check_every)
      return cfdb_fail(e->ctx, CFDB_ENUMERIC, "cfdb_euler_run: the clock did not reach t_end within max_steps");
  }
  if (steps_done) *steps_done = steps;
  if (final_in_b) *final_in_b = int(steps & 1);
  return CFDB_OK;
}
