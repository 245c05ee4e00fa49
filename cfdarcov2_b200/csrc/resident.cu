// Cluster-resident heat solver for meshes small enough to live in on-chip
// memory: the whole field stays in the distributed shared memory (two
// buffers) of one thread-block cluster of up to 16 CTAs, or of up to four
// such clusters, every time step runs inside ONE launch and the steps are
// separated by the cluster barrier instead of a kernel boundary.  The CTAs
// split x into consecutive slabs; each thread updates 4 consecutive z cells
// (one float4) per group.
//
//  * heat_resident_k, one cluster: CTA c owns the x slab
//    [c X / CL, (c+1) X / CL); the x neighbours of a slab's first and last
//    planes are read from the adjacent CTAs' shared memory (distributed
//    shared memory loads), everything else is local.
//  * heat_resident_multi_k, G clusters (fields too large for one): each CTA
//    keeps its slab's two x neighbour planes in halo slots of its own shared
//    memory, which the neighbouring CTAs of its cluster fill with remote
//    stores as they compute their edge planes (so every read of a step is
//    local); across two clusters the edge plane goes through global memory
//    (L2) behind a release/acquire step counter that the reading CTA polls
//    with a bounded wait.  Only the CTAs at a cluster's edge wait, and only
//    for their two neighbours: there is no grid-wide barrier.
//
// A step of a 64^3 mesh through the per-step TMA sweep costs ~4 us, almost
// all of it launch and pipeline fill; here a step is one pass over shared
// memory plus one cluster barrier (and, with several clusters, one plane
// handed across each cluster boundary).  The cell update is heat_update(),
// the same function the sweep uses, so the paths round identically.
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
constexpr int kMaxClusters = 4;  // clusters side by side along x
constexpr int kErrResidentTimeout = 1;  // the device error word's wait-timeout code

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

struct MultiArgs {
  int X, Y, Z;
  int P;  // planes per buffer (the largest slab)
  int steps;
  int G;  // clusters
  float cx, cy, cz;
  // the first (side 0) and last (side 1) plane of every cluster's range
  // after each step, by step parity ([G][2][2][Y Z] floats), and the steps
  // published per cluster side ([G][2], zero before the launch)
  float* xb;
  unsigned long long* done;
  long long wait_cycles;
  int* err;
  int skip_step;  // test hook (>= 0): cluster 1 does not publish its planes of this step
};

__device__ __forceinline__ unsigned long long ld_acquire_gpu(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// Waits until *p >= v, at most `limit` SM clock cycles.
__device__ __forceinline__ bool wait_counter(const unsigned long long* p, unsigned long long v, long long limit) {
  if (ld_acquire_gpu(p) >= v) return true;
  const long long t0 = clock64();
  while (ld_acquire_gpu(p) < v)
    if (clock64() - t0 > limit) return false;
  return true;
}

__global__ void __launch_bounds__(kThreads, 1)
    heat_resident_multi_k(const float* __restrict__ in, float* __restrict__ out, MultiArgs a) {
  extern __shared__ __align__(16) float sm[];
  cg::cluster_group cl = cg::this_cluster();
  const int c = int(cl.block_rank());
  const int CL = int(cl.num_blocks());
  const int g = int(blockIdx.x) / CL;
  const int NB = CL * a.G;
  const int b = g * CL + c;
  auto slab_start = [&](int blk) { return int((long long)blk * a.X / NB); };
  const int x0 = slab_start(b), x1 = slab_start(b + 1);
  const int np = x1 - x0;
  const int plane = a.Y * a.Z;
  // a buffer holds the slab's planes at positions 1 .. np and the x
  // neighbours' planes x0 - 1 and x1 at positions 0 and np + 1 (halo slots)
  const int buf = (a.P + 2) * plane;
  const int zq = a.Z / 4;
  const int groups = np * a.Y * zq;
  const int tid = int(threadIdx.x);

  // the slab and its halo planes into buffer 0
  {
    const int lo_x = x0 > 0 ? x0 - 1 : x0, hi_x = x1 < a.X ? x1 : x1 - 1;
    const float4* src = reinterpret_cast<const float4*>(in + (long long)x0 * plane);
    float4* dst = reinterpret_cast<float4*>(sm + plane);
    for (int i = tid; i < np * plane / 4; i += kThreads) dst[i] = src[i];
    const float4* slo = reinterpret_cast<const float4*>(in + (long long)lo_x * plane);
    const float4* shi = reinterpret_cast<const float4*>(in + (long long)hi_x * plane);
    float4* dlo = reinterpret_cast<float4*>(sm);
    float4* dhi = reinterpret_cast<float4*>(sm + (np + 1) * plane);
    for (int i = tid; i < plane / 4; i += kThreads) {
      dlo[i] = slo[i];
      dhi[i] = shi[i];
    }
  }
  // this thread's groups, one word each: offset within the plane (bits
  // 0-14), plane of the slab (bits 15-22) and flags (bits 23-30): x / y / z
  // walls below and above (1, 2 / 4, 8 / 16, 32), first and last plane of
  // the slab (64, 128); -1 for no group
  int code[kMaxGroups];
#pragma unroll
  for (int k = 0; k < kMaxGroups; ++k) {
    const int gi = tid + k * kThreads;
    code[k] = -1;
    if (gi < groups) {
      const int p = gi / (a.Y * zq);
      const int r = gi - p * (a.Y * zq);
      const int y = r / zq;
      const int z = 4 * (r - y * zq);
      const int f = (x0 + p == 0 ? 1 : 0) | (x0 + p == a.X - 1 ? 2 : 0) | (y == 0 ? 4 : 0) | (y == a.Y - 1 ? 8 : 0) |
                    (z == 0 ? 16 : 0) | (z + 4 == a.Z ? 32 : 0) | (p == 0 ? 64 : 0) | (p == np - 1 ? 128 : 0);
      code[k] = (y * a.Z + z) | (p << 15) | (f << 23);
    }
  }
  // Inside a cluster each CTA writes its new first and last planes into the
  // halo slots of the neighbouring CTAs (distributed shared memory stores,
  // made visible by the cluster barrier), so every read of a step is local.
  // Across two clusters the cluster's first / last plane is published in
  // global memory (L2) behind a step counter, and the neighbouring cluster's
  // edge CTA reads it from there after a bounded wait.
  const bool lo_dsm = c > 0, hi_dsm = c < CL - 1;
  const bool lo_ext = !lo_dsm && g > 0, hi_ext = !hi_dsm && g < a.G - 1;
  float* nlo = lo_dsm ? cl.map_shared_rank(sm, c - 1) : nullptr;
  float* nhi = hi_dsm ? cl.map_shared_rank(sm, c + 1) : nullptr;
  const int nlo_hi_slot = lo_dsm ? (x0 - slab_start(b - 1) + 1) * plane : 0;  // the lower CTA's slot of plane x0
  const bool pub_lo = lo_ext, pub_hi = hi_ext;
  auto xplane = [&](int cluster, int side, int parity) {
    return a.xb + ((size_t(cluster) * 2 + side) * 2 + parity) * size_t(plane);
  };
  bool waits_ok = true;
  cl.sync();

  for (int s = 0; s < a.steps; ++s) {
    const float* A = sm + (s & 1) * buf;
    float* B = sm + ((s + 1) & 1) * buf;
    const int nb = ((s + 1) & 1) * buf;  // buffer s + 1 in a neighbour's shared memory
    const bool ext = s > 0 && (lo_ext || hi_ext);  // before the first step the halo slots hold the input planes
    const float* Xlo = lo_ext ? xplane(g - 1, 1, s & 1) : nullptr;
    const float* Xhi = hi_ext ? xplane(g + 1, 0, s & 1) : nullptr;
    if (ext) {
      // one thread waits until the neighbouring clusters published step s;
      // after the barrier every thread of the CTA reads those planes (from
      // L2: ld.global.cg, so no stale L1 line of two steps ago is used)
      if (tid == 0 && waits_ok) {
        if (lo_ext) waits_ok = wait_counter(a.done + (g - 1) * 2 + 1, (unsigned long long)s, a.wait_cycles);
        if (hi_ext && waits_ok) waits_ok = wait_counter(a.done + (g + 1) * 2 + 0, (unsigned long long)s, a.wait_cycles);
        if (!waits_ok) atomicExch(a.err, kErrResidentTimeout);
      }
      __syncthreads();
    }
    float* plo = pub_lo ? xplane(g, 0, (s + 1) & 1) : nullptr;
    float* phi = pub_hi ? xplane(g, 1, (s + 1) & 1) : nullptr;
#pragma unroll
    for (int k = 0; k < kMaxGroups; ++k) {
      if (code[k] < 0) continue;
      const int yz = code[k] & 0x7fff, f = code[k] >> 23;
      const int o = (((code[k] >> 15) & 0xff) + 1) * plane + yz;
      const float4 C = *reinterpret_cast<const float4*>(A + o);
      float4 XM, XP;
      if (f & 1) XM = C;
      else if (ext && lo_ext && (f & 64)) XM = __ldcg(reinterpret_cast<const float4*>(Xlo + yz));
      else XM = *reinterpret_cast<const float4*>(A + o - plane);
      if (f & 2) XP = C;
      else if (ext && hi_ext && (f & 128)) XP = __ldcg(reinterpret_cast<const float4*>(Xhi + yz));
      else XP = *reinterpret_cast<const float4*>(A + o + plane);
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
      if (f & 64) {
        if (lo_dsm) *reinterpret_cast<float4*>(nlo + nb + nlo_hi_slot + yz) = R;
        else if (pub_lo) __stcg(reinterpret_cast<float4*>(plo + yz), R);
      }
      if (f & 128) {
        if (hi_dsm) *reinterpret_cast<float4*>(nhi + nb + yz) = R;
        else if (pub_hi) __stcg(reinterpret_cast<float4*>(phi + yz), R);
      }
    }
    if ((pub_lo || pub_hi) && s + 1 < a.steps) {
      // the published planes complete before the step counter moves on
      __threadfence();
      __syncthreads();
      if (tid == 0 && !(g == 1 && a.skip_step >= 0 && s + 1 >= a.skip_step)) {
        if (pub_lo) st_release_gpu(a.done + g * 2 + 0, (unsigned long long)(s + 1));
        if (pub_hi) st_release_gpu(a.done + g * 2 + 1, (unsigned long long)(s + 1));
      }
    }
    cl.sync();  // step s written everywhere (halo slots included), and nobody reads buffer s & 1 any more
  }

  // the final state to global memory
  {
    const float4* src = reinterpret_cast<const float4*>(sm + (a.steps & 1) * buf + plane);
    float4* dst = reinterpret_cast<float4*>(out + (long long)x0 * plane);
    for (int i = tid; i < np * plane / 4; i += kThreads) dst[i] = src[i];
  }
}

}  // namespace

namespace {

cudaLaunchConfig_t cluster_config(cfdb_ctx* ctx, long long blocks, int CL, long long smem, cudaLaunchAttribute* attr,
                                  bool cooperative) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(unsigned(blocks));
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = size_t(smem);
  cfg.stream = ctx->stream;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = unsigned(CL);
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  attr[1].id = cudaLaunchAttributeCooperative;
  attr[1].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = cooperative ? 2 : 1;
  return cfg;
}

// One cluster holds the field (heat_resident_k).
int run_single(cfdb_ctx* ctx, cfdb_mesh* m, const void* Ta, void* Tb, double k, double dt, int32_t steps,
               int max_smem, int* launched) {
  const long long plane = m->ny * m->nz;
  for (int CL = std::min<long long>(kMaxCluster, m->nx); CL >= 2; CL /= 2) {
    const long long P = (m->nx + CL - 1) / CL;
    const long long smem = 2 * P * plane * 4;
    if (smem > max_smem) break;  // fewer CTAs only make the slabs larger
    if (P * plane / 4 > (long long)kMaxGroups * kThreads) continue;
    // per-device kernel attribute; cheap enough to set on every call
    CFDB_CUDA(ctx, cudaFuncSetAttribute(heat_resident_k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    CFDB_CUDA(ctx, cudaFuncSetAttribute(heat_resident_k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    cudaLaunchAttribute attr[2];
    cudaLaunchConfig_t cfg = cluster_config(ctx, CL, CL, smem, attr, false);
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

// G co-resident clusters hold the field (heat_resident_multi_k), as one
// cooperative launch.
int run_multi(cfdb_ctx* ctx, cfdb_mesh* m, const void* Ta, void* Tb, double k, double dt, int32_t steps, int G,
              int max_smem, int* launched) {
  const long long plane = m->ny * m->nz;
  for (int CL = std::min<long long>(kMaxCluster, m->nx); CL >= 2; CL /= 2) {
    const long long NB = (long long)G * CL;
    if (NB > m->nx) continue;
    const long long P = (m->nx + NB - 1) / NB;
    const long long smem = 2 * (P + 2) * plane * 4;
    if (smem > max_smem) break;
    if (P * plane / 4 > (long long)kMaxGroups * kThreads || P > 256) continue;  // the group words' fields
    CFDB_CUDA(ctx, cudaFuncSetAttribute(heat_resident_multi_k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    CFDB_CUDA(ctx, cudaFuncSetAttribute(heat_resident_multi_k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    cudaLaunchAttribute attr[2];
    cudaLaunchConfig_t cfg = cluster_config(ctx, NB, CL, smem, attr, true);
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, heat_resident_multi_k, &cfg) != cudaSuccess || clusters < G) {
      cudaGetLastError();
      continue;
    }
    MultiArgs a;
    a.X = int(m->nx); a.Y = int(m->ny); a.Z = int(m->nz);
    a.P = int(P);
    a.steps = steps;
    a.G = G;
    a.cx = float(dt * k / (m->dx * m->dx));
    a.cy = float(dt * k / (m->dy * m->dy));
    a.cz = float(dt * k / (m->dz * m->dz));
    a.wait_cycles = ctx->wait_cycles;
    a.err = ctx->d_error;
    a.skip_step = ctx->missing_plane;
    void* ws = nullptr;
    const size_t xb_bytes = size_t(G) * 4 * size_t(plane) * 4;
    if (int rc = cfdb_ws_alloc(ctx, int64_t(xb_bytes + size_t(G) * 2 * 8), &ws)) return rc;
    a.xb = static_cast<float*>(ws);
    a.done = reinterpret_cast<unsigned long long*>(static_cast<char*>(ws) + xb_bytes);
    cudaError_t e = cudaMemsetAsync(a.done, 0, size_t(G) * 2 * 8, ctx->stream);
    float* out = static_cast<float*>((steps & 1) ? Tb : const_cast<void*>(Ta));
    if (e == cudaSuccess) e = cudaLaunchKernelEx(&cfg, heat_resident_multi_k, static_cast<const float*>(Ta), out, a);
    cfdb_ws_free(ctx, ws);
    if (e != cudaSuccess) {
      cudaGetLastError();  // a cooperative launch of this size is refused: the caller tries fewer clusters
      continue;
    }
    ++ctx->launches;
    *launched = int(NB);
    return CFDB_OK;
  }
  return CFDB_EUNSUPPORTED;
}

}  // namespace

// Runs `steps` heat steps in one launch when the mesh fits the shared memory
// of one cluster, else of kMaxClusters (or half as many) co-resident
// clusters; returns CFDB_EUNSUPPORTED (nothing launched, no error recorded)
// otherwise, and the caller takes the per-step path.  One cluster comes
// first: handing a plane across clusters costs about 1.7 us per step (the
// fence, the counter and its poll through L2), so a 64^3 step on four
// clusters (3.35 us) gains next to nothing over one (3.1 us), while a field
// too large for one cluster (128 x 64 x 64 on four) runs 3.9 us per step
// against 5.5-6.2 on the per-step path.  Several clusters run as one
// cooperative launch, which either makes every CTA resident at once or
// fails (then fewer clusters are tried), so a CTA never waits on a cluster
// that has not started.  The result goes to Tb for odd `steps`, else to
// Ta, as with the ping-pong of the per-step path; the other buffer is left
// as it was.
int heat_resident_run(cfdb_ctx* ctx, cfdb_mesh* m, const void* Ta, void* Tb, double k, double dt, int32_t steps,
                      int* launched) {
  *launched = 0;
  if (!m->uniform || m->nz % 4 != 0 || steps < 1) return CFDB_EUNSUPPORTED;
  if ((reinterpret_cast<uintptr_t>(Ta) | reinterpret_cast<uintptr_t>(Tb)) & 15u) return CFDB_EUNSUPPORTED;
  int max_smem = 0;
  CFDB_CUDA(ctx, cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
  int rc = run_single(ctx, m, Ta, Tb, k, dt, steps, max_smem, launched);
  for (int G = kMaxClusters; rc == CFDB_EUNSUPPORTED && G >= 2; G /= 2)
    rc = run_multi(ctx, m, Ta, Tb, k, dt, steps, G, max_smem, launched);
  return rc;
}
