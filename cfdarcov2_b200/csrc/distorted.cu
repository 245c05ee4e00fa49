// Fused acoustic step on vertex (distorted) meshes.  Geometry is the compact
// FP32 form built by cfdb_mesh_need_compact: per cell the outward area
// vectors S = n_alt A of its +x/+y/+z faces and 1/V (40 B/cell) on a lattice
// padded below each axis; the -faces are the minus neighbours' +faces negated
// (the reference computes one normal and one area per face object and gives
// the two cells opposite outward normals, src/mesh3d.cpp:69-105), and on the
// -walls that neighbour is a ghost entry holding the wall face's vector.
// Warps cover consecutive z cells, so every neighbour gather is a coalesced
// row segment.
#include "tma_host.hpp"

CFDB_MODULE_ANCHOR

namespace {

constexpr int kThreads = 256;

struct CompactArgs {
  const float* __restrict__ S;  // padded compact geometry, 10 fields of np entries
  long long np, yp, zp;
  int X, Y, Z;
  long long n;
};

// Approximate (SFU) square root and reciprocal in their flush-to-zero
// forms: |S| and 1/|S|^2 of faces, which are never subnormal; the IEEE
// sequences would add fix-up paths, and the division a slow path for
// subnormal numerators (the far tails of a smooth pulse).
__device__ __forceinline__ float face_sqrt(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float face_rcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__global__ void __launch_bounds__(kThreads)
    compact_wave_k(CompactArgs g, const float* __restrict__ q, float* __restrict__ qn, const float* __restrict__ cf,
                   float cconst, int mode, float dt) {
  const long long n = g.n;
  const long long yz = (long long)g.Y * g.Z;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = int(i / yz);
    const int rem = int(i - (long long)x * yz);
    const int y = rem / g.Z;
    const int z = rem - y * g.Z;
    const float pP = q[i], uP = q[n + i], vP = q[2 * n + i], wP = q[3 * n + i];
    const float cP = cf ? cf[i] : cconst;
    const float c2 = cP * cP;
    float ap = 0.f, au = 0.f, av = 0.f, aw = 0.f;
    const long long stride[3] = {yz, (long long)g.Z, 1};
    const long long pi = ((long long)(x + 1) * g.yp + (y + 1)) * g.zp + (z + 4);  // padded geometry entry
    const long long pstride[3] = {g.yp * g.zp, g.zp, 1};
    const int coord[3] = {x, y, z};
    const int ext[3] = {g.X, g.Y, g.Z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        float Sx, Sy, Sz;
        bool wall;
        long long j;
        if (side == 1) {  // +face: own area vector
          Sx = g.S[(3 * d + 0) * g.np + pi]; Sy = g.S[(3 * d + 1) * g.np + pi]; Sz = g.S[(3 * d + 2) * g.np + pi];
          wall = coord[d] == ext[d] - 1;
          j = i + stride[d];
        } else {          // -face: the minus neighbour's (or the wall ghost's) +face negated
          wall = coord[d] == 0;
          j = i - stride[d];
          const long long pj = pi - pstride[d];
          Sx = -g.S[(3 * d + 0) * g.np + pj]; Sy = -g.S[(3 * d + 1) * g.np + pj]; Sz = -g.S[(3 * d + 2) * g.np + pj];
        }
        const float S2 = Sx * Sx + Sy * Sy + Sz * Sz;
        const float A = face_sqrt(S2);
        const float unPA = uP * Sx + vP * Sy + wP * Sz;
        float pN, uN, vN, wN, cN;
        if (!wall) {
          pN = q[j]; uN = q[n + j]; vN = q[2 * n + j]; wN = q[3 * n + j];
          cN = cf ? cf[j] : cconst;
        } else {
          const float k2 = 2.f * unPA * face_rcp(S2);  // reflect about the unit normal S/A
          pN = pP; uN = uP - k2 * Sx; vN = vP - k2 * Sy; wN = wP - k2 * Sz; cN = cP;
        }
        const float unNA = uN * Sx + vN * Sy + wN * Sz;
        const float cfc = mode == 0 ? fmaxf(cP, cN) : 0.5f * (cP + cN);
        const float hA = 0.5f * cfc * A;
        const float pm = 0.5f * (pP + pN);
        ap += c2 * 0.5f * (unPA + unNA) - hA * (pN - pP);
        au += pm * Sx - hA * (uN - uP);
        av += pm * Sy - hA * (vN - vP);
        aw += pm * Sz - hA * (wN - wP);
      }
    }
    const float s = -dt * g.S[9 * g.np + pi];
    qn[i] = pP + s * ap;
    qn[n + i] = uP + s * au;
    qn[2 * n + i] = vP + s * av;
    qn[3 * n + i] = wP + s * aw;
  }
}

// Face-flux form (face_sweep.cuh): the flux through a face is evaluated once
// and enters the two cells it separates with opposite signs.  The face with
// normal e_d between L (minus side) and R carries L's +d area vector S, and
//   F = ( c^2/2 (u_L + u_R).S - c|S|/2 (p_R - p_L),
//         (p_L + p_R)/2 S     - c|S|/2 (u_R - u_L) )
// is what the gather form adds to L (and subtracts from R): the same terms as
// compact_wave_k per face (constant c, where both speed modes agree), summed
// as F(+d) - F(-d) per direction.  A wall face reflects the cell's velocity
// about the face normal (the cell's own +d vector, or on a -wall the ghost
// entry's vector, which is the wall face's outward vector negated).
struct DistFacePhys {
  static constexpr int NF = 4;
  static constexpr int NG = 10;  // [S+x | S+y | S+z | 1/V]
  static constexpr int NGF = 3;
  static constexpr int ND = 0;
  // the reflection costs a division: evaluate wall faces behind a branch
  static constexpr bool SELECT_WALLS = false;
  static constexpr int MIN_BLOCKS = 2;
  struct Params {
    float dt, c2h, hc;  // dt, c^2/2, c/2
  };
  struct Acc {};
  // |S| of a face: the PTX approximate square root (relative error ~2^-22,
  // far inside the FP32 path's 1e-5 bar) in its flush-to-zero form (|S|^2 of
  // any face longer than ~1e-9 is far above FP32's smallest normal)
  __device__ static float fast_sqrt(float x) { return face_sqrt(x); }
  __device__ static float fast_rcp(float x) { return face_rcp(x); }
  __device__ static bool begin(Params&) { return true; }
  __device__ static void flux(const float L[NF], const float*, const float R[NF], const float*, const float S[NGF],
                              int, const Params& a, float F[NF]) {
    const float A = fast_sqrt(S[0] * S[0] + S[1] * S[1] + S[2] * S[2]);
    const float unL = L[1] * S[0] + L[2] * S[1] + L[3] * S[2];
    const float unR = R[1] * S[0] + R[2] * S[1] + R[3] * S[2];
    const float hA = a.hc * A;
    const float pm = 0.5f * (L[0] + R[0]);
    F[0] = a.c2h * (unL + unR) - hA * (R[0] - L[0]);
    F[1] = pm * S[0] - hA * (R[1] - L[1]);
    F[2] = pm * S[1] - hA * (R[2] - L[2]);
    F[3] = pm * S[2] - hA * (R[3] - L[3]);
  }
  // The cell beyond a wall face with area vector S: the cell with its
  // velocity reflected about the face normal.  1/|S|^2 by the approximate
  // reciprocal: an IEEE division takes a slow path for a subnormal
  // numerator, which the far tails of a smooth pulse produce, and with it
  // stalls every warp holding a wall face (12 % of a step on a Gaussian
  // pulse).
  __device__ static void ghost(const float C[NF], const float*, const float S[NGF], int, float g[NF], float*) {
    const float k2 =
        2.f * (C[1] * S[0] + C[2] * S[1] + C[3] * S[2]) * fast_rcp(S[0] * S[0] + S[1] * S[1] + S[2] * S[2]);
    g[0] = C[0];
    g[1] = C[1] - k2 * S[0];
    g[2] = C[2] - k2 * S[1];
    g[3] = C[3] - k2 * S[2];
  }
  __device__ static void update(const float C[NF], const float*, const float G[NG], const float dF[3][NF],
                                const Params& a, float o[NF]) {
    const float s = -a.dt * G[9];
#pragma unroll
    for (int f = 0; f < NF; ++f) o[f] = C[f] + s * (dF[0][f] + dF[1][f] + dF[2][f]);
  }
  __device__ static void acc_init(Acc&) {}
  __device__ static void acc_cell(Acc&, const float*, const Params&) {}
  __device__ static void finish(Acc&, const Params&, bool) {}
};

}  // namespace

int compact_wave_step(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* q, void* qn, const void* c, double cconst,
                      int mode, double dt) {
  if (dtype != CFDB_F32)
    return cfdb_fail(ctx, CFDB_EUNSUPPORTED, "the fused vertex-mesh wave step computes in float32 only");
  if (int rc = cfdb_mesh_need_compact(m)) return rc;
  const CompactGeomDev& cg = m->compact;
  if (!c && m->nz % 4 == 0 && !(reinterpret_cast<uintptr_t>(q) & 15u) && !(reinterpret_cast<uintptr_t>(qn) & 15u)) {
    const float cs = float(cconst);
    const DistFacePhys::Params p{float(dt), 0.5f * cs * cs, 0.5f * cs};
    const stencil::PaddedGeom pg{cg.S, cg.zp, cg.yp, m->nx + 1, cg.np};
    // 64-wide z tiles (two cells per thread) unless 32-wide ones pad the z rows less
    const int64_t pad64 = (m->nz + 63) / 64 * 64 - m->nz, pad32 = (m->nz + 31) / 32 * 32 - m->nz;
    if (m->nz > 32 && pad64 <= pad32) return stencil::launch_face_sweep<DistFacePhys, 64, 8, 3, 2>(ctx, m, q, pg, qn, p, 0);
    return stencil::launch_face_sweep<DistFacePhys, 32, 8, 3, 1>(ctx, m, q, pg, qn, p, 0);
  }
  CompactArgs a{cg.S, cg.np, cg.yp, cg.zp, int(m->nx), int(m->ny), int(m->nz), (long long)m->n};
  compact_wave_k<<<grid_for(ctx, m->n, kThreads, 8), kThreads, 0, ctx->stream>>>(
      a, static_cast<const float*>(q), static_cast<float*>(qn), static_cast<const float*>(c), float(cconst), mode,
      float(dt));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}
