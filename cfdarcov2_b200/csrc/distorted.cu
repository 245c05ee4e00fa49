// Fused acoustic step on vertex (distorted) meshes.  Geometry is the compact
// FP32 form built by cfdb_mesh_need_compact: per cell the outward area
// vectors S = n_alt A of its +x/+y/+z faces and 1/V (40 B/cell); the -faces
// are the neighbours' +faces negated (the reference computes one normal and
// one area per face object and gives the two cells opposite outward normals,
// src/mesh3d.cpp:69-105), boundary -faces come from three wall tables.
// Warps cover consecutive z cells, so every neighbour gather is a coalesced
// row segment.
#include "tma_host.hpp"

CFDB_MODULE_ANCHOR

namespace {

constexpr int kThreads = 256;

struct CompactArgs {
  const float* __restrict__ S;
  const float* __restrict__ iv;
  const float* __restrict__ wx;
  const float* __restrict__ wy;
  const float* __restrict__ wz;
  int X, Y, Z;
  long long n;
};

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
          Sx = g.S[(3 * d + 0) * n + i]; Sy = g.S[(3 * d + 1) * n + i]; Sz = g.S[(3 * d + 2) * n + i];
          wall = coord[d] == ext[d] - 1;
          j = i + stride[d];
        } else {          // -face: neighbour's +face negated, or the wall table
          wall = coord[d] == 0;
          j = i - stride[d];
          if (!wall) {
            Sx = -g.S[(3 * d + 0) * n + j]; Sy = -g.S[(3 * d + 1) * n + j]; Sz = -g.S[(3 * d + 2) * n + j];
          } else {
            const float* w = d == 0 ? g.wx : (d == 1 ? g.wy : g.wz);
            const long long cnt = d == 0 ? yz : (d == 1 ? (long long)g.X * g.Z : (long long)g.X * g.Y);
            const long long k = d == 0 ? (long long)y * g.Z + z : (d == 1 ? (long long)x * g.Z + z : (long long)x * g.Y + y);
            Sx = w[k]; Sy = w[cnt + k]; Sz = w[2 * cnt + k];
          }
        }
        const float A = sqrtf(Sx * Sx + Sy * Sy + Sz * Sz);
        const float unPA = uP * Sx + vP * Sy + wP * Sz;
        float pN, uN, vN, wN, cN;
        if (!wall) {
          pN = q[j]; uN = q[n + j]; vN = q[2 * n + j]; wN = q[3 * n + j];
          cN = cf ? cf[j] : cconst;
        } else {
          const float k2 = 2.f * unPA / (A * A);  // reflect about the unit normal S/A
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
    const float s = -dt * g.iv[i];
    qn[i] = pP + s * ap;
    qn[n + i] = uP + s * au;
    qn[2 * n + i] = vP + s * av;
    qn[3 * n + i] = wP + s * aw;
  }
}

// Sweep form (uniform-lattice topology, any vertex positions): the state
// (p,u,v,w) is swept, the compact geometry [Sx|Sy|Sz|1/V] (10 fields) is
// staged as auxiliary data with the same halos, so the -face area vector of a
// cell is its staged neighbour's +face vector.  -wall faces read the wall
// tables.  Same flux as compact_wave_k.
struct DistPhys {
  // |S| of a face: the PTX approximate square root (relative error ~2^-22,
  // far inside the FP32 path's 1e-5 bar) instead of the IEEE sequence
  __device__ static float fast_sqrt(float x) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
  }
  static constexpr int NF = 4;
  static constexpr int NA = 10;
  static constexpr bool HAS_C = false;
  static constexpr int FT = 14;
  static constexpr int MIN_BLOCKS = 3;
  struct Params {
    float dt, c;
    int mode;
    int X, Y, Z;
    const float* wx;
    const float* wy;
    const float* wz;
  };
  struct Acc {};
  __device__ static bool begin(Params&) { return true; }
  __device__ static void ghost(float g[FT], const float p[FT], int) {
#pragma unroll
    for (int f = 0; f < FT; ++f) g[f] = p[f];
  }
  __device__ static void cell(const stencil::CellIn<FT>& in, const Params& a, float o[NF]) {
    const float* P = in.P;
    const float pP = P[0], uP = P[1], vP = P[2], wP = P[3];
    const float cP = a.c, c2 = cP * cP;
    float ap = 0.f, au = 0.f, av = 0.f, aw = 0.f;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const int k = 2 * d + side;
        const bool wall = (in.walls >> k) & 1;
        float Sx, Sy, Sz;
        if (side) {
          Sx = P[4 + 3 * d]; Sy = P[5 + 3 * d]; Sz = P[6 + 3 * d];
        } else if (!wall) {
          const float* N = in.nb[k];
          Sx = -N[4 + 3 * d]; Sy = -N[5 + 3 * d]; Sz = -N[6 + 3 * d];
        } else {
          const long long yz = (long long)a.Y * a.Z;
          const int x = int(in.idx / yz);
          const int r = int(in.idx - (long long)x * yz);
          const int y = r / a.Z, z = r - (r / a.Z) * a.Z;
          const float* w = d == 0 ? a.wx : (d == 1 ? a.wy : a.wz);
          const long long cnt = d == 0 ? yz : (d == 1 ? (long long)a.X * a.Z : (long long)a.X * a.Y);
          const long long kk = d == 0 ? (long long)y * a.Z + z : (d == 1 ? (long long)x * a.Z + z : (long long)x * a.Y + y);
          Sx = w[kk]; Sy = w[cnt + kk]; Sz = w[2 * cnt + kk];
        }
        const float A = fast_sqrt(Sx * Sx + Sy * Sy + Sz * Sz);
        const float unPA = uP * Sx + vP * Sy + wP * Sz;
        float pN, uN, vN, wN;
        if (!wall) {
          const float* N = in.nb[k];
          pN = N[0]; uN = N[1]; vN = N[2]; wN = N[3];
        } else {
          const float k2 = 2.f * unPA / (A * A);
          pN = pP; uN = uP - k2 * Sx; vN = vP - k2 * Sy; wN = wP - k2 * Sz;
        }
        const float unNA = uN * Sx + vN * Sy + wN * Sz;
        const float hA = 0.5f * cP * A;
        const float pm = 0.5f * (pP + pN);
        ap += c2 * 0.5f * (unPA + unNA) - hA * (pN - pP);
        au += pm * Sx - hA * (uN - uP);
        av += pm * Sy - hA * (vN - vP);
        aw += pm * Sz - hA * (wN - wP);
      }
    }
    const float s = -a.dt * P[13];
    o[0] = pP + s * ap;
    o[1] = uP + s * au;
    o[2] = vP + s * av;
    o[3] = wP + s * aw;
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
    DistPhys::Params p{float(dt), float(cconst), mode, int(m->nx), int(m->ny), int(m->nz), cg.wall_x, cg.wall_y, cg.wall_z};
    return stencil::launch_sweep<DistPhys, 32, 8, 3, 1>(ctx, m, q, cg.S, nullptr, qn, p, 0);
  }
  CompactArgs a{cg.S, cg.inv_vol, cg.wall_x, cg.wall_y, cg.wall_z, int(m->nx), int(m->ny), int(m->nz), (long long)m->n};
  compact_wave_k<<<grid_for(ctx, m->n, kThreads, 8), kThreads, 0, ctx->stream>>>(
      a, static_cast<const float*>(q), static_cast<float*>(qn), static_cast<const float*>(c), float(cconst), mode,
      float(dt));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}
