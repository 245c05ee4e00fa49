// Cluster-resident heat solver for meshes small enough to live in on-chip
// memory: one thread-block cluster of up to 16 CTAs holds the whole field in
// its distributed shared memory (two buffers), runs every time step in ONE
// launch and synchronises the steps with the cluster barrier instead of a
// kernel boundary.  CTA c owns the x slab [c X / CL, (c+1) X / CL); the x
// neighbours of a slab's first and last planes are read from the adjacent
// CTAs' shared memory (distributed shared memory loads), everything else is
// local.  Each thread updates 4 consecutive z cells (one float4) per group.
//
// A step of a 64^3 mesh through the per-step TMA sweep costs ~4 us, almost
// all of it launch and pipeline fill; here a step is one pass over shared
// memory plus one cluster barrier.  The cell update is heat_update(), the
// same function the sweep uses, so the two paths round identically.
#include <cooperative_groups.h>

#include <algorithm>

#include "cfdb_internal.hpp"
#include "heat_cell.cuh"

CFDB_MODULE_ANCHOR

namespace cg = cooperative_groups;

namespace {

constexpr int kThreads = 1024;
constexpr int kMaxGroups = 8;   // float4 groups per thread and step
constexpr int kMaxCluster = 16;  // non-portable cluster size

struct ResidentArgs {
  int X, Y, Z;
  int P;  // planes per buffer (the largest slab)
  int steps;
  float cx, cy, cz;
};

__global__ void __launch_bounds__(kThreads, 1)
    heat_resident_k(const float* __restrict__ in, float* __restrict__ out, ResidentArgs a) {
  extern __shared__ __align__(16) float sm[];
  cg::cluster_group cl = cg::this_cluster();
  const int c = int(cl.block_rank());
  const int CL = int(cl.num_blocks());
  const int x0 = int((long long)c * a.X / CL), x1 = int((long long)(c + 1) * a.X / CL);
  const int np = x1 - x0;
  const int plane = a.Y * a.Z;
  const int buf = a.P * plane;  // floats per buffer
  const int zq = a.Z / 4;
  const int groups = np * a.Y * zq;
  const int tid = int(threadIdx.x);

  // the slab into buffer 0
  {
    const float4* src = reinterpret_cast<const float4*>(in + (long long)x0 * plane);
    float4* dst = reinterpret_cast<float4*>(sm);
    for (int i = tid; i < np * plane / 4; i += kThreads) dst[i] = src[i];
  }
  // this thread's groups: offset in a buffer, offset within the plane and
  // which neighbours are walls
  int off[kMaxGroups], inpl[kMaxGroups], flags[kMaxGroups];
#pragma unroll
  for (int k = 0; k < kMaxGroups; ++k) {
    const int g = tid + k * kThreads;
    off[k] = -1;
    inpl[k] = 0;
    flags[k] = 0;
    if (g < groups) {
      const int p = g / (a.Y * zq);
      const int r = g - p * (a.Y * zq);
      const int y = r / zq;
      const int z = 4 * (r - y * zq);
      inpl[k] = y * a.Z + z;
      off[k] = p * plane + inpl[k];
      flags[k] = (p == 0 ? 1 : 0) | (p == np - 1 ? 2 : 0) | (y == 0 ? 4 : 0) | (y == a.Y - 1 ? 8 : 0) |
                 (z == 0 ? 16 : 0) | (z + 4 == a.Z ? 32 : 0);
    }
  }
  // neighbour slabs' shared memory (the plane next to ours in each)
  const float* lo = c > 0 ? cl.map_shared_rank(sm, c - 1) : sm;
  const float* hi = c < CL - 1 ? cl.map_shared_rank(sm, c + 1) : sm;
  const int lo_plane = c > 0 ? (x0 - 1) - int((long long)(c - 1) * a.X / CL) : 0;
  cl.sync();

  for (int s = 0; s < a.steps; ++s) {
    const float* A = sm + (s & 1) * buf;
    float* B = sm + ((s + 1) & 1) * buf;
    const float* Alo = lo + (s & 1) * buf + lo_plane * plane;  // x0 - 1 in the lower slab
    const float* Ahi = hi + (s & 1) * buf;                      // x1 in the upper slab
#pragma unroll
    for (int k = 0; k < kMaxGroups; ++k) {
      if (off[k] < 0) continue;
      const int o = off[k], f = flags[k], yz = inpl[k];
      const float4 C = *reinterpret_cast<const float4*>(A + o);
      float4 XM, XP;
      if (!(f & 1)) XM = *reinterpret_cast<const float4*>(A + o - plane);
      else if (c > 0) XM = *reinterpret_cast<const float4*>(Alo + yz);
      else XM = C;
      if (!(f & 2)) XP = *reinterpret_cast<const float4*>(A + o + plane);
      else if (c < CL - 1) XP = *reinterpret_cast<const float4*>(Ahi + yz);
      else XP = C;
      const float4 YM = (f & 4) ? C : *reinterpret_cast<const float4*>(A + o - a.Z);
      const float4 YP = (f & 8) ? C : *reinterpret_cast<const float4*>(A + o + a.Z);
      const float zl = (f & 16) ? C.x : A[o - 1];
      const float zr = (f & 32) ? C.w : A[o + 4];
      float4 R;
      R.x = heat_update(C.x, XM.x, XP.x, YM.x, YP.x, zl, C.y, a.cx, a.cy, a.cz);
      R.y = heat_update(C.y, XM.y, XP.y, YM.y, YP.y, C.x, C.z, a.cx, a.cy, a.cz);
      R.z = heat_update(C.z, XM.z, XP.z, YM.z, YP.z, C.y, C.w, a.cx, a.cy, a.cz);
      R.w = heat_update(C.w, XM.w, XP.w, YM.w, YP.w, C.z, zr, a.cx, a.cy, a.cz);
      *reinterpret_cast<float4*>(B + o) = R;
    }
    cl.sync();  // step s written everywhere, and nobody reads buffer s & 1 any more
  }

  // the final state to global memory
  {
    const float4* src = reinterpret_cast<const float4*>(sm + (a.steps & 1) * buf);
    float4* dst = reinterpret_cast<float4*>(out + (long long)x0 * plane);
    for (int i = tid; i < np * plane / 4; i += kThreads) dst[i] = src[i];
  }
}

}  // namespace

// Runs `steps` heat steps in one cluster launch when the mesh fits; returns
// CFDB_EUNSUPPORTED (nothing launched, no error recorded) otherwise, and the
// caller takes the per-step path.  The result goes to Tb for odd `steps`,
// else to Ta, as with the ping-pong of the per-step path; the other buffer
// is left as it was.
int heat_resident_run(cfdb_ctx* ctx, cfdb_mesh* m, const void* Ta, void* Tb, double k, double dt, int32_t steps,
                      int* launched) {
  *launched = 0;
  if (!m->uniform || m->nz % 4 != 0 || steps < 1) return CFDB_EUNSUPPORTED;
  if ((reinterpret_cast<uintptr_t>(Ta) | reinterpret_cast<uintptr_t>(Tb)) & 15u) return CFDB_EUNSUPPORTED;
  const long long plane = m->ny * m->nz;
  int max_smem = 0;
  CFDB_CUDA(ctx, cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
  for (int CL = std::min<long long>(kMaxCluster, m->nx); CL >= 2; CL /= 2) {
    const long long P = (m->nx + CL - 1) / CL;
    const long long smem = 2 * P * plane * 4;
    if (smem > max_smem) break;  // fewer CTAs only make the slabs larger
    if (P * plane / 4 > (long long)kMaxGroups * kThreads) continue;
    // per-device kernel attribute; cheap enough to set on every call
    CFDB_CUDA(ctx, cudaFuncSetAttribute(heat_resident_k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    CFDB_CUDA(ctx, cudaFuncSetAttribute(heat_resident_k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(CL);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = size_t(smem);
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = unsigned(CL);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, heat_resident_k, &cfg) != cudaSuccess || clusters < 1) {
      cudaGetLastError();
      continue;
    }
    ResidentArgs a;
    a.X = int(m->nx); a.Y = int(m->ny); a.Z = int(m->nz);
    a.P = int(P);
    a.steps = steps;
    a.cx = float(dt * k / (m->dx * m->dx));
    a.cy = float(dt * k / (m->dy * m->dy));
    a.cz = float(dt * k / (m->dz * m->dz));
    float* out = static_cast<float*>((steps & 1) ? Tb : const_cast<void*>(Ta));
    CFDB_CUDA(ctx, cudaLaunchKernelEx(&cfg, heat_resident_k, static_cast<const float*>(Ta), out, a));
    ++ctx->launches;
    *launched = CL;
    return CFDB_OK;
  }
  return CFDB_EUNSUPPORTED;
}
