// Discrete adjoint of the acoustic step on uniform meshes (speed_mode 1,
// c_f = (c_P + c_N)/2), FP32.  With q' = q + dt A(c) q the reverse step is
//   lam  = lam' + dt A(c)^T lam'
//   g_c += dt (d(A(c) q)/dc)^T lam'
// A^T is applied as a gather: each cell collects the flux sensitivities of
// its six faces from both sides, so no scatter or atomics are needed.  Uses
// the volume-scaled adjoint lt = lam / V (R(N) carries 1/V_N).  The same
// arithmetic on the general geometry is plain_ops.cu's wave_adjoint_plain_k.
#include "f32x2.cuh"
#include "tma_host.hpp"

CFDB_MODULE_ANCHOR

namespace {

constexpr int kThreads = 256;

// TMA-sweep form of the same adjoint step: lam (4 fields) is the swept state,
// the forward state q_n (4 fields) is staged as auxiliary data and c as the
// coefficient field, all with their halos; the c-gradient of each cell is
// accumulated in place.
struct AdjPhys {
  static constexpr int NF = 4;
  static constexpr int NA = 4;
  static constexpr bool HAS_C = true;
  static constexpr int FT = 9;
  static constexpr int MIN_BLOCKS = 2;
  struct Params {
    float A[3];   // face areas normal to x, y, z
    float A2[3];  // A / 2
    float A4[3];  // A / 4
    float iV;     // 1 / cell volume
    float dt;
    float* gc;
  };
  struct Acc {};
  __device__ static bool begin(Params&) { return true; }
  // dJ/dc of the cell so far: loaded by the sweep one plane ahead (in.pre)
  static constexpr bool HAS_PRE = true;
  __device__ static float* pre_ptr(const Params& a) { return a.gc; }
  // Reflective wall, as in the forward step: the ghost mirrors the
  // wall-normal component of lam and of q and copies c.  With it the
  // interior face terms below reproduce the wall terms of the transposed
  // forward step exactly (ap -= s A lam_d, au_d -= c_P A lam_d,
  // gg -= A q_d lam_d), so no face needs a branch.
  __device__ static void ghost(float g[FT], const float p[FT], int dir) {
#pragma unroll
    for (int f = 0; f < FT; ++f) g[f] = p[f];
    g[1 + dir] = -p[1 + dir];
    g[5 + dir] = -p[5 + dir];
  }
  // Per face with outward normal s e_d, area A and neighbour N (dl = lam_N -
  // lam_P, dq = q_N - q_P, all 4 fields; h = A (c_P + c_N) / 4):
  //   ap   += h dl_p + s A/2 dl_d
  //   au_e += h dl_e,   au_d += s A/2 (c_N^2 lam_N,p - c_P^2 lam_P,p)
  //   gg   -= s A c_P (2 q_P,d + dq_d) lam_P,p + A/4 sum_f dq_f dl_f
  // The s-odd terms of the two faces of one direction (neighbours M at -d,
  // N at +d) collapse into central differences:
  //   ap   += A/2 (lam_N,d - lam_M,d)
  //   au_d += A/2 (c_N^2 lam_N,p - c_M^2 lam_M,p)
  //   gg   -= c_P lam_P,p A (q_N,d - q_M,d)
  // leaving the h and dq.dl terms per face.  Every term is linear in lam / V
  // with one uniform V, so 1/V multiplies the sums once at the end.
  __device__ static void cell(const stencil::CellIn<FT>& in, const Params& a, float o[NF]) {
    const float g0 = in.pre;
    const float* P = in.P;
    const float cP = P[8];
    float ap = 0.f, au[3] = {0.f, 0.f, 0.f}, gq = 0.f, gw = 0.f;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float* M = in.nb[2 * d];
      const float* N = in.nb[2 * d + 1];
      float w = 0.f;
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const float* X = side ? N : M;
        const float h = a.A4[d] * (cP + X[8]);
        const float dl0 = X[0] - P[0], dl1 = X[1] - P[1], dl2 = X[2] - P[2], dl3 = X[3] - P[3];
        const float dq0 = X[4] - P[4], dq1 = X[5] - P[5], dq2 = X[6] - P[6], dq3 = X[7] - P[7];
        ap += h * dl0;
        au[0] += h * dl1;
        au[1] += h * dl2;
        au[2] += h * dl3;
        w += (dq0 * dl0 + dq1 * dl1) + (dq2 * dl2 + dq3 * dl3);
      }
      ap += a.A2[d] * (N[1 + d] - M[1 + d]);
      au[d] += a.A2[d] * (N[8] * N[8] * N[0] - M[8] * M[8] * M[0]);
      gq += a.A[d] * (N[5 + d] - M[5 + d]);
      gw += a.A4[d] * w;
    }
    const float gg = -(cP * P[0]) * gq - gw;
    const float s = a.dt * a.iV;
    o[0] = P[0] + s * ap;
    o[1] = P[1] + s * au[0];
    o[2] = P[2] + s * au[1];
    o[3] = P[3] + s * au[2];
    a.gc[in.idx] = g0 + s * gg;
  }
  // The same update for the thread's two cells at once (the sweep runs two
  // z cells per thread): every value is a (cell 0, cell 1) pair and every
  // operation one packed f32x2 instruction, halving the FP32 instruction
  // count of the issue-bound step.
  static constexpr bool PAIRED = true;
  __device__ static void cell2(const stencil::CellIn<FT>& i0, const stencil::CellIn<FT>& i1, const Params& a,
                               float o0[NF], float o1[NF]) {
    using namespace f2;
    auto pr = [](float u, float v) { return make_float2(u, v); };
    float2 P[FT];
#pragma unroll
    for (int f = 0; f < FT; ++f) P[f] = pr(i0.P[f], i1.P[f]);
    const float2 cP = P[8];
    float2 ap = splat(0.f), au[3] = {splat(0.f), splat(0.f), splat(0.f)}, gq = splat(0.f), gw = splat(0.f);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      float2 M[FT], N[FT];
#pragma unroll
      for (int f = 0; f < FT; ++f) {
        M[f] = pr(i0.nb[2 * d][f], i1.nb[2 * d][f]);
        N[f] = pr(i0.nb[2 * d + 1][f], i1.nb[2 * d + 1][f]);
      }
      const float2 A4 = splat(a.A4[d]), A2 = splat(a.A2[d]);
      float2 w = splat(0.f);
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const float2* X = side ? N : M;
        const float2 h = mul(A4, add(cP, X[8]));
        const float2 dl0 = sub(X[0], P[0]), dl1 = sub(X[1], P[1]), dl2 = sub(X[2], P[2]), dl3 = sub(X[3], P[3]);
        const float2 dq0 = sub(X[4], P[4]), dq1 = sub(X[5], P[5]), dq2 = sub(X[6], P[6]), dq3 = sub(X[7], P[7]);
        ap = fma(h, dl0, ap);
        au[0] = fma(h, dl1, au[0]);
        au[1] = fma(h, dl2, au[1]);
        au[2] = fma(h, dl3, au[2]);
        w = add(w, add(fma(dq1, dl1, mul(dq0, dl0)), fma(dq3, dl3, mul(dq2, dl2))));
      }
      ap = fma(A2, sub(N[1 + d], M[1 + d]), ap);
      au[d] = fma(A2, sub(mul(mul(N[8], N[8]), N[0]), mul(mul(M[8], M[8]), M[0])), au[d]);
      gq = fma(splat(a.A[d]), sub(N[5 + d], M[5 + d]), gq);
      gw = fma(A4, w, gw);
    }
    const float2 gg = sub(neg(mul(mul(cP, P[0]), gq)), gw);
    const float2 s = splat(a.dt * a.iV);
    const float2 r0 = fma(s, ap, P[0]), r1 = fma(s, au[0], P[1]), r2 = fma(s, au[1], P[2]), r3 = fma(s, au[2], P[3]);
    const float2 gn = fma(s, gg, pr(i0.pre, i1.pre));
    o0[0] = r0.x; o1[0] = r0.y;
    o0[1] = r1.x; o1[1] = r1.y;
    o0[2] = r2.x; o1[2] = r2.y;
    o0[3] = r3.x; o1[3] = r3.y;
    // the two cells are consecutive in z: one 8-byte store (idx even: z tiles start at multiples of 2)
    if ((i0.idx & 1) == 0) {
      *reinterpret_cast<float2*>(a.gc + i0.idx) = gn;
    } else {
      a.gc[i0.idx] = gn.x;
      a.gc[i1.idx] = gn.y;
    }
  }
  __device__ static void acc_init(Acc&) {}
  __device__ static void acc_cell(Acc&, const float*, const Params&) {}
  __device__ static void finish(Acc&, const Params&, bool) {}
};

struct AdjArgs {
  int X, Y, Z;
  long long n;
  float A[3];  // face areas normal to x, y, z
  float iV;    // 1 / cell volume
  float dt;
};

__global__ void __launch_bounds__(kThreads)
    wave_adjoint_k(AdjArgs a, const float* __restrict__ q, const float* __restrict__ lam1, float* __restrict__ lam0,
                   const float* __restrict__ cf, float* __restrict__ gc) {
  const long long n = a.n;
  const long long yz = (long long)a.Y * a.Z;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = int(i / yz);
    const int rem = int(i - (long long)x * yz);
    const int y = rem / a.Z;
    const int z = rem - y * a.Z;
    const int coord[3] = {x, y, z};
    const int ext[3] = {a.X, a.Y, a.Z};
    const long long stride[3] = {yz, (long long)a.Z, 1};
    const float cP = cf[i];
    float lP[4], qP[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      lP[f] = lam1[f * n + i] * a.iV;
      qP[f] = q[f * n + i];
    }
    float ap = 0.f, au[3] = {0.f, 0.f, 0.f}, gg = 0.f;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float A = a.A[d];
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const float s = side ? 1.f : -1.f;  // outward normal = s e_d
        const bool wall = side ? (coord[d] == ext[d] - 1) : (coord[d] == 0);
        if (!wall) {
          const long long j = side ? i + stride[d] : i - stride[d];
          const float cN = cf[j];
          float lN[4], qN[4];
#pragma unroll
          for (int f = 0; f < 4; ++f) {
            lN[f] = lam1[f * n + j] * a.iV;
            qN[f] = q[f * n + j];
          }
          const float h = 0.25f * (cP + cN) * A;
          ap += h * (lN[0] - lP[0]) + 0.5f * s * A * (lN[1 + d] - lP[1 + d]);
          const float sp = 0.5f * (cN * cN * lN[0] - cP * cP * lP[0]);
#pragma unroll
          for (int e = 0; e < 3; ++e) au[e] += h * (lN[1 + e] - lP[1 + e]);
          au[d] += sp * s * A;
          gg -= cP * s * A * (qP[1 + d] + qN[1 + d]) * lP[0];
          const float jp = qN[0] - qP[0];
          float ju_self = 0.f, ju_nb = 0.f;
#pragma unroll
          for (int e = 0; e < 3; ++e) {
            ju_self += (qN[1 + e] - qP[1 + e]) * lP[1 + e];
            ju_nb += (qP[1 + e] - qN[1 + e]) * lN[1 + e];
          }
          gg += 0.25f * A * ((jp * lP[0] + ju_self) + (ju_nb - jp * lN[0]));
        } else {
          ap -= s * A * lP[1 + d];
          au[d] -= cP * A * lP[1 + d];
          gg -= A * qP[1 + d] * lP[1 + d];
        }
      }
    }
    lam0[i] = lam1[i] + a.dt * ap;
#pragma unroll
    for (int e = 0; e < 3; ++e) lam0[(1 + e) * n + i] = lam1[(1 + e) * n + i] + a.dt * au[e];
    gc[i] += a.dt * gg;
  }
}

}  // namespace

int fused_wave_adjoint(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* q, const void* lam1, void* lam0,
                       const void* c, void* gc, double dt) {
  (void)dtype;
  if (stencil::check_sweep(ctx, m, {q, lam1, lam0, c, gc}) == CFDB_OK) {
    AdjPhys::Params p;
    p.A[0] = float(m->dy * m->dz); p.A[1] = float(m->dx * m->dz); p.A[2] = float(m->dx * m->dy);
    for (int d = 0; d < 3; ++d) {
      p.A2[d] = 0.5f * p.A[d];
      p.A4[d] = 0.25f * p.A[d];
    }
    p.iV = float(1.0 / (m->dx * m->dy * m->dz));
    p.dt = float(dt);
    p.gc = static_cast<float*>(gc);
    if (m->nz >= 64) return stencil::launch_sweep<AdjPhys, 64, 8, 4, 2>(ctx, m, lam1, q, c, lam0, p, 0);
    return stencil::launch_sweep<AdjPhys, 32, 8, 4, 2>(ctx, m, lam1, q, c, lam0, p, 0);
  }
  // shapes the sweep cannot stage (nz % 4 != 0 or unaligned pointers): gather form
  AdjArgs a;
  a.X = int(m->nx); a.Y = int(m->ny); a.Z = int(m->nz);
  a.n = (long long)m->n;
  a.A[0] = float(m->dy * m->dz); a.A[1] = float(m->dx * m->dz); a.A[2] = float(m->dx * m->dy);
  a.iV = float(1.0 / (m->dx * m->dy * m->dz));
  a.dt = float(dt);
  wave_adjoint_k<<<grid_for(ctx, m->n, kThreads, 8), kThreads, 0, ctx->stream>>>(
      a, static_cast<const float*>(q), static_cast<const float*>(lam1), static_cast<float*>(lam0),
      static_cast<const float*>(c), static_cast<float*>(gc));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}
