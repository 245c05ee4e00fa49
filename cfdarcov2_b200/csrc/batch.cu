// Batched ensemble of independent small problems (cubes of n^3 cells on
// [0,1]^3, heat or the acoustic wave system) advanced together: one
// persistent launch per step walks a table of work items (problem, a run of
// `threads` (y, z) columns, a range of x planes) covering about
// `cells_per_item` cells each; every thread marches one column along x.
// Per-problem constants (dt, k or c, spacing) live in a device table, so
// uneven sizes and parameters share one kernel; the step is replayed from a
// captured CUDA graph.  cells_per_item, the CTA size and the CTAs per SM are
// chosen by an autotuner that times candidates on the real pools and caches
// the winner per device and problem set.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include <unistd.h>

#include "cfdb_internal.hpp"
#include "tma_stencil.cuh"

CFDB_MODULE_ANCHOR

namespace {

struct ProbDev {
  int32_t n;
  int32_t kind;
  float c0, c1, c2;  // heat: c0 = dt k / dx^2; wave: c0 = dt c^2 / (2 dx), c1 = dt c / (2 dx), c2 = dt / (2 dx)
  int64_t offset;
};

// A work item: `threads` consecutive (y, z) columns (yz0, yz0 + 1, ...) of
// one problem, marched over the x planes [x0, x1).  Each thread decodes its
// (y, z) once, keeps the x neighbours of its column in registers (previous /
// current / next plane) and reads the y and z neighbours of the current
// plane through L1 (the CTA's own columns, contiguous in z).  Measured
// alternatives: items of whole rows leave more threads idle (1.4x slower);
// staging each plane in shared memory needs a barrier per plane, which
// exposes the load latency of every plane (2x slower); prefetching columns
// four planes ahead into L2 gained nothing and added DRAM reads; loading
// plane x + 2 into registers one iteration early (two planes in flight per
// warp) was 8 % slower (items of the tuned size march only 8 planes); two
// heat columns per thread (two independent load chains) changed nothing, nor
// did fetching the next item's descriptors while the current item marches.
struct ItemDev {
  int32_t prob;
  int32_t yz0;
  int32_t x0, x1;
};

// One step of one work item: every thread with a cell marches its (y, z)
// column over the item's planes.  NF = 1 (heat: T' = T + c0 sum_faces
// (T_N - T), zero-gradient walls) or 4 (the acoustic system with constant c:
// Rusanov dissipation = weighted Laplacian, reflective walls).  A wall
// neighbour is the cell itself, for the wave with its wall-normal velocity
// negated.  No barriers: warps run ahead independently, which keeps many
// plane loads in flight.
template <int NF>
__device__ __forceinline__ void column_step(const ProbDev& P, const ItemDev& I, const float* __restrict__ a,
                                            float* __restrict__ b) {
  const int n = P.n, n2 = n * n;
  const int64_t n3 = int64_t(n2) * n;
  const int col = I.yz0 + int(threadIdx.x);  // the thread's column within a plane
  if (col >= n2) return;
  const int y = col / n;
  const int z = col - y * n;
  // One pointer per field to the column's cell in the current plane,
  // advanced by a plane per step of the march; the y neighbours sit at a
  // fixed offset from it (or at the cell itself on a wall) and the z
  // neighbours at +-1, read unconditionally and replaced by the cell itself
  // on a wall (the pool keeps spare floats before its first and after its
  // last problem, so those reads stay inside it).
  const float* q[NF];
  float* o[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    q[f] = a + P.offset + f * n3 + int64_t(I.x0) * n2 + col;
    o[f] = b + P.offset + f * n3 + int64_t(I.x0) * n2 + col;
  }
  const int dym = y > 0 ? -n : 0, dyp = y < n - 1 ? n : 0;
  const bool zlo = z == 0, zhi = z == n - 1;
  const float sym = y > 0 ? 1.f : -1.f, syp = y < n - 1 ? 1.f : -1.f;
  const float szm = zlo ? -1.f : 1.f, szp = zhi ? -1.f : 1.f;
  float cur[NF], prv[NF], nxt[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) cur[f] = __ldg(q[f]);
  if (I.x0 > 0) {
#pragma unroll
    for (int f = 0; f < NF; ++f) prv[f] = __ldg(q[f] - n2);
  } else {
#pragma unroll
    for (int f = 0; f < NF; ++f) prv[f] = cur[f];
    if constexpr (NF == 4) prv[1] = -cur[1];
  }
  for (int x = I.x0; x < I.x1; ++x) {
    const float* qn[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) qn[f] = q[f] + n2;
    if (x + 1 < n) {
#pragma unroll
      for (int f = 0; f < NF; ++f) nxt[f] = __ldg(qn[f]);
    } else {
#pragma unroll
      for (int f = 0; f < NF; ++f) nxt[f] = cur[f];
      if constexpr (NF == 4) nxt[1] = -cur[1];
    }
    float ym[NF], yp[NF], zm[NF], zp[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      ym[f] = __ldg(q[f] + dym);
      yp[f] = __ldg(q[f] + dyp);
      const float l = __ldg(q[f] - 1), r = __ldg(q[f] + 1);
      zm[f] = zlo ? cur[f] : l;
      zp[f] = zhi ? cur[f] : r;
    }
    if constexpr (NF == 1) {
      const float t = cur[0];
      const float s = ((prv[0] - t) + (nxt[0] - t)) + ((ym[0] - t) + (yp[0] - t)) + ((zm[0] - t) + (zp[0] - t));
      *o[0] = t + P.c0 * s;
    } else {
      ym[2] *= sym;
      yp[2] *= syp;
      zm[3] *= szm;
      zp[3] *= szp;
      // p' = p - c0 div(u) + c1 lapl(p);  u_e' = u_e - c2 d_e(p) + c1 lapl(u_e)
      // (central differences over the face pairs, lapl = sum of the six
      // neighbours - 6 x the cell: a cube with one spacing)
      float s[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) s[f] = ((prv[f] + nxt[f]) + (ym[f] + yp[f])) + (zm[f] + zp[f]);
      const float div = ((nxt[1] - prv[1]) + (yp[2] - ym[2])) + (zp[3] - zm[3]);
      *o[0] = cur[0] - P.c0 * div + P.c1 * (s[0] - 6.0f * cur[0]);
      *o[1] = cur[1] - P.c2 * (nxt[0] - prv[0]) + P.c1 * (s[1] - 6.0f * cur[1]);
      *o[2] = cur[2] - P.c2 * (yp[0] - ym[0]) + P.c1 * (s[2] - 6.0f * cur[2]);
      *o[3] = cur[3] - P.c2 * (zp[0] - zm[0]) + P.c1 * (s[3] - 6.0f * cur[3]);
    }
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      prv[f] = cur[f];
      cur[f] = nxt[f];
      q[f] = qn[f];
      o[f] += n2;
    }
  }
}

// Heat columns carry one field, so a thread marching one column has a
// single load chain in flight; with two columns per thread (heat items are
// twice as wide: columns yz0 + t and yz0 + t + blockDim.x) the two marches
// interleave and twice the loads are in flight.  Same arithmetic per cell.
__device__ __forceinline__ void heat_columns2(const ProbDev& P, const ItemDev& I, const float* __restrict__ a,
                                              float* __restrict__ b) {
  const int n = P.n, n2 = n * n;
  int colv[2] = {I.yz0 + int(threadIdx.x), I.yz0 + int(threadIdx.x) + int(blockDim.x)};
  const bool act[2] = {colv[0] < n2, colv[1] < n2};
  if (!act[0]) return;
  const float* q[2];
  float* o[2];
  int dym[2], dyp[2];
  bool zlo[2], zhi[2];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const int col = act[c] ? colv[c] : colv[0];  // an idle second column shadows the first
    const int y = col / n, z = col - (col / n) * n;
    q[c] = a + P.offset + int64_t(I.x0) * n2 + col;
    o[c] = b + P.offset + int64_t(I.x0) * n2 + col;
    dym[c] = y > 0 ? -n : 0;
    dyp[c] = y < n - 1 ? n : 0;
    zlo[c] = z == 0;
    zhi[c] = z == n - 1;
  }
  float cur[2], prv[2], nxt[2];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    cur[c] = __ldg(q[c]);
    prv[c] = I.x0 > 0 ? __ldg(q[c] - n2) : cur[c];
  }
  for (int x = I.x0; x < I.x1; ++x) {
    const float* qn[2] = {q[0] + n2, q[1] + n2};
    float ym[2], yp[2], zm[2], zp[2];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      nxt[c] = x + 1 < n ? __ldg(qn[c]) : cur[c];
      ym[c] = __ldg(q[c] + dym[c]);
      yp[c] = __ldg(q[c] + dyp[c]);
      const float l = __ldg(q[c] - 1), r = __ldg(q[c] + 1);
      zm[c] = zlo[c] ? cur[c] : l;
      zp[c] = zhi[c] ? cur[c] : r;
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const float t = cur[c];
      const float s = ((prv[c] - t) + (nxt[c] - t)) + ((ym[c] - t) + (yp[c] - t)) + ((zm[c] - t) + (zp[c] - t));
      if (act[c]) *o[c] = t + P.c0 * s;
      prv[c] = cur[c];
      cur[c] = nxt[c];
      q[c] = qn[c];
      o[c] += n2;
    }
  }
}

// One launch per step walks the work items.  Two register budgets: 64
// (MINB = 1), or 48 for blocks of up to 256 threads (no spills), where 40
// warps fit an SM instead of 32 and more plane loads are in flight -- faster
// for heat-only batches (260 against 312 us per step at 512 cubes), slower
// for the mixed heat/wave set, so the tuner picks.
template <int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) batch_step_k(const ProbDev* __restrict__ probs, const ItemDev* __restrict__ items, int n_items,
                             const float* __restrict__ a, float* __restrict__ b, int heat_cols) {
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const ItemDev I = items[it];
    const ProbDev P = probs[I.prob];
    if (P.kind == 1) column_step<4>(P, I, a, b);
    else if (heat_cols == 2) heat_columns2(P, I, a, b);
    else column_step<1>(P, I, a, b);
  }
}

// ---- staged form: a producer warp streams plane rows into a shared ring -----
//
// The same work items and arithmetic as column_step, with the planes staged
// in shared memory.  Warp 0 is the producer: its lane 0 walks the CTA's
// items and, for every plane an item needs (x0 - 1 .. x1), issues one 1-D
// bulk copy (cp.async.bulk, no multicast) per field of the contiguous rows
// [yz0 - n, yz0 + C + n) of that plane -- the item's C columns and their y
// neighbours -- into ring slot k % S, completing on the slot's `full`
// mbarrier.  The remaining warps are consumers: each thread owns one column
// of the item, takes its own cell and its y/z neighbours from the slot, keeps
// the x neighbours in registers, and its warp arrives on the slot's `empty`
// mbarrier when done with the plane; the producer refills a slot once every
// consumer warp has released it.  No CTA-wide barrier per plane, and the
// ring runs on across item boundaries, so up to S planes stay in flight per
// CTA.  Copies start on a 16-byte boundary (rounded down; the consumer skips
// the 0-3 leading floats) and end on one (rounded up: the pool holds 4 spare
// floats at its end).  Every wait is bounded; a wait that gives up records
// the timeout in the error word, skips the remaining waits, and the producer
// lets its copies land before the CTA exits.
// Ring depth S (slots): 8 where the shared memory of the configured CTAs
// holds it, else 4 (ring_slots()).

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   stencil::smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(stencil::smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(stencil::smem_u32(bar)) : "memory");
}

struct RingArgs {
  int C;                  // consumer threads = columns per item
  int cap;                // floats per field tile of a slot (multiple of 4)
  long long wait_cycles;  // bound of every mbarrier wait
};

template <int NF, uint32_t S>
__device__ __forceinline__ void ring_consume(const ProbDev& P, const ItemDev& I, const float* __restrict__ ring,
                                             uint64_t* full, uint64_t* empty, const RingArgs& A,
                                             float* __restrict__ b, uint32_t& k, bool& bad) {
  static_assert((S & (S - 1)) == 0, "ring slots: a power of two");
  const int n = P.n, n2 = n * n;
  const int n3 = n2 * n;  // n <= 1024
  const int t = int(threadIdx.x) - 32;
  const int col = I.yz0 + t;
  const bool act = col < n2;
  const int lo = max(I.yz0 - n, 0);
  const int y = act ? col / n : 0;
  const int z = act ? col - y * n : 0;
  const int j = col - lo;  // the thread's cell in a slot's row block, before the alignment shift
  const int dym = y > 0 ? -n : 0, dyp = y < n - 1 ? n : 0, dzm = z > 0 ? -1 : 0, dzp = z < n - 1 ? 1 : 0;
  const float sym = y > 0 ? 1.f : -1.f, syp = y < n - 1 ? 1.f : -1.f;
  const float szm = z > 0 ? 1.f : -1.f, szp = z < n - 1 ? 1.f : -1.f;
  const unsigned lane = threadIdx.x & 31u;
  // Field f of plane x starts its copy at the 16-byte boundary below
  // element P.offset + f n3 + x n2 + lo, so the thread's cell sits at
  // j + ((P.offset + f n3 + x n2 + lo) & 3): the shift is tracked mod 4.
  const int s0 = int((P.offset + lo) & 3), fs = n3 & 3, xs = n2 & 3;
  auto off = [&](uint32_t kk, int f, int x) {
    return int(kk & (S - 1)) * (4 * A.cap) + f * A.cap + ((s0 + f * fs + x * xs) & 3) + j;
  };
  auto wait_full = [&](uint32_t kk) {
    if (!bad && !stencil::mbar_wait_bounded(&full[kk & (S - 1)], (kk / S) & 1u, A.wait_cycles)) bad = true;
  };
  auto release = [&](uint32_t kk) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[kk & (S - 1)]);
  };
  auto ghost = [&](float g[NF], const float c[NF]) {
#pragma unroll
    for (int f = 0; f < NF; ++f) g[f] = c[f];
    if constexpr (NF == 4) g[1] = -c[1];
  };
  float prv[NF], cur[NF], nxt[NF];
  if (I.x0 > 0) {
    wait_full(k);
    if (act) {
#pragma unroll
      for (int f = 0; f < NF; ++f) prv[f] = ring[off(k, f, I.x0 - 1)];
    }
    release(k);
    ++k;
  }
  wait_full(k);
  if (act) {
#pragma unroll
    for (int f = 0; f < NF; ++f) cur[f] = ring[off(k, f, I.x0)];
  }
  uint32_t kc = k++;
  if (I.x0 == 0) ghost(prv, cur);
  float* const o = b + P.offset + col;  // field f of plane x: o[f n3 + x n2]
  for (int x = I.x0; x < I.x1; ++x) {
    uint32_t kn = kc;
    if (x + 1 < n) {
      wait_full(k);
      if (act) {
#pragma unroll
        for (int f = 0; f < NF; ++f) nxt[f] = ring[off(k, f, x + 1)];
      }
      kn = k++;
    } else {
      ghost(nxt, cur);
    }
    if (act) {
      float ym[NF], yp[NF], zm[NF], zp[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const float* q = ring + off(kc, f, x);
        ym[f] = q[dym];
        yp[f] = q[dyp];
        zm[f] = q[dzm];
        zp[f] = q[dzp];
      }
      const int c = x * n2;
      if constexpr (NF == 1) {
        const float tt = cur[0];
        const float sum = ((prv[0] - tt) + (nxt[0] - tt)) + ((ym[0] - tt) + (yp[0] - tt)) + ((zm[0] - tt) + (zp[0] - tt));
        o[c] = tt + P.c0 * sum;
      } else {
        ym[2] *= sym;
        yp[2] *= syp;
        zm[3] *= szm;
        zp[3] *= szp;
        float sm[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) sm[f] = ((prv[f] + nxt[f]) + (ym[f] + yp[f])) + (zm[f] + zp[f]);
        const float div = ((nxt[1] - prv[1]) + (yp[2] - ym[2])) + (zp[3] - zm[3]);
        o[c] = cur[0] - P.c0 * div + P.c1 * (sm[0] - 6.0f * cur[0]);
        o[n3 + c] = cur[1] - P.c2 * (nxt[0] - prv[0]) + P.c1 * (sm[1] - 6.0f * cur[1]);
        o[2 * n3 + c] = cur[2] - P.c2 * (yp[0] - ym[0]) + P.c1 * (sm[2] - 6.0f * cur[2]);
        o[3 * n3 + c] = cur[3] - P.c2 * (zp[0] - zm[0]) + P.c1 * (sm[3] - 6.0f * cur[3]);
      }
    }
    release(kc);
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      prv[f] = cur[f];
      cur[f] = nxt[f];
    }
    kc = kn;
  }
  if (I.x1 < n) release(kc);  // plane x1, loaded as the last plane's x+1 neighbour
}

template <int S>
__global__ void batch_ring_k(const ProbDev* __restrict__ probs, const ItemDev* __restrict__ items, int n_items,
                             const float* __restrict__ a, float* __restrict__ b, RingArgs A, int* __restrict__ err) {
  extern __shared__ __align__(128) float ring[];
  __shared__ __align__(8) uint64_t full[S], empty[S];
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      stencil::mbar_init(&full[s], 1);
      stencil::mbar_init(&empty[s], blockDim.x / 32 - 1);
    }
    stencil::fence_mbar_init();
  }
  __syncthreads();
  bool bad = false;
  if (threadIdx.x < 32) {
    // Producer warp: lane s < S owns ring slot s and issues every plane
    // that lands there (global plane index k with k % S == s), so the lanes
    // prepare up to S planes per warp instruction and wait on their own
    // slots independently.
    const uint32_t lane = threadIdx.x;
    uint32_t k = 0;        // planes of the CTA's earlier items
    int64_t last = -1;     // the last plane this lane issued
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
      const ItemDev I = items[it];
      const ProbDev P = probs[I.prob];
      const int n = P.n, n2 = n * n;
      const int64_t n3 = int64_t(n2) * n;
      const int nf = P.kind == 0 ? 1 : 4;
      const int lo = max(I.yz0 - n, 0), hi = min(I.yz0 + A.C + n, n2);
      const int xb = max(I.x0 - 1, 0), xe = min(I.x1, n - 1);
      const int np = xe - xb + 1;
      if (lane < uint32_t(S) && !bad) {
        const int64_t base = P.offset + lo;
        for (int q = int((lane - k) & uint32_t(S - 1)); q < np; q += S) {
          const uint32_t kk = k + uint32_t(q);  // kk % S == lane
          // refill the slot only when every consumer warp has released its
          // previous plane and that plane's copies have landed (the latter
          // holds whenever the consumers waited for them; checking it keeps
          // the slot's barrier from being armed over an unfinished phase)
          if (kk >= uint32_t(S) &&
              (!stencil::mbar_wait_bounded(&empty[lane], ((kk / S) - 1) & 1u, A.wait_cycles) ||
               !stencil::mbar_wait_bounded(&full[lane], ((kk / S) - 1) & 1u, A.wait_cycles))) {
            bad = true;
            break;
          }
          const int64_t plane = base + int64_t(xb + q) * n2;
          int64_t g0[4];
          uint32_t bytes[4], total = 0;
          for (int f = 0; f < nf; ++f) {
            const int64_t start = plane + f * n3;
            g0[f] = start & ~int64_t(3);
            const int64_t end = (start + (hi - lo) + 3) & ~int64_t(3);
            bytes[f] = uint32_t(4 * (end - g0[f]));
            total += bytes[f];
          }
          float* dst = ring + lane * (4 * A.cap);
          stencil::mbar_expect_tx(&full[lane], total);
          for (int f = 0; f < nf; ++f) bulk_g2s(dst + f * A.cap, a + g0[f], bytes[f], &full[lane]);
          last = kk;
        }
      }
      k += uint32_t(np);
    }
    // let every copy this lane issued land before the CTA exits (immediate
    // unless a consumer gave up): the slot's last copy is its newest phase
    if (last >= 0 && !stencil::mbar_wait_bounded(&full[lane], (uint32_t(last) / S) & 1u, A.wait_cycles)) bad = true;
  } else {
    uint32_t k = 0;
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
      const ItemDev I = items[it];
      const ProbDev P = probs[I.prob];
      if (P.kind == 0) ring_consume<1, uint32_t(S)>(P, I, ring, full, empty, A, b, k, bad);
      else ring_consume<4, uint32_t(S)>(P, I, ring, full, empty, A, b, k, bad);
    }
  }
  if (bad) atomicExch(err, stencil::kErrWaitTimeout);
}

}  // namespace

constexpr int64_t kPoolPad = 4;  // spare floats before the first and after the last problem of a pool
// kernel forms (cfdb_batch_set_staged)
constexpr int kFormMarch = 0, kFormRing = 1, kFormMarch48 = 2;

struct cfdb_batch {
  cfdb_ctx* ctx = nullptr;
  int nmax = 0;  // largest n of the problem set
  std::vector<cfdb_problem> probs;
  int64_t pool = 0;
  ProbDev* d_probs = nullptr;
  ItemDev* d_items = nullptr;
  int n_items = 0;
  int items_cap = 0;
  int cells_per_item = 2048, threads = 256, ctas_per_sm = 4;
  int staged = kFormMarch;  // kernel form (kForm*); the tuner picks the fastest
  int heat_cols = 1;        // columns per thread of the heat items in the item table (2 for the march forms)
  int ring_resident = 0;          // CTAs of the staged kernel one SM holds
  int64_t ring_resident_key = -1;  // (threads, shared bytes) ring_resident was measured for
  int64_t last_launches = 0;
  cudaGraphExec_t graph = nullptr;
  const void* graph_a = nullptr;
  const void* graph_b = nullptr;
  int graph_cfg[3] = {0, 0, 0};
};

namespace {

int build_items(cfdb_batch* b) {
  // runs of `threads` columns x `planes` x planes, planes = cells_per_item / threads
  std::vector<ItemDev> items;
  const int planes = std::max(1, b->cells_per_item / b->threads);
  const int heat_cols = b->staged == kFormRing ? 1 : 2;
  for (size_t p = 0; p < b->probs.size(); ++p) {
    const int n = b->probs[p].n;
    // heat items of the column march cover two columns per thread
    const int width = b->probs[p].kind == 0 ? heat_cols * b->threads : b->threads;
    for (int yz0 = 0; yz0 < n * n; yz0 += width)
      for (int x0 = 0; x0 < n; x0 += planes) items.push_back(ItemDev{int32_t(p), yz0, x0, std::min(n, x0 + planes)});
  }
  if (int(items.size()) > b->items_cap) {
    cfdb_dev_free(b->ctx, b->d_items);
    b->d_items = nullptr;
    if (int rc = cfdb_dev_alloc(b->ctx, int64_t(sizeof(ItemDev)) * items.size(), reinterpret_cast<void**>(&b->d_items)))
      return rc;
    b->items_cap = int(items.size());
  }
  CFDB_CUDA(b->ctx, cudaMemcpy(b->d_items, items.data(), sizeof(ItemDev) * items.size(), cudaMemcpyHostToDevice));
  b->n_items = int(items.size());
  b->heat_cols = heat_cols;
  return CFDB_OK;
}

void drop_graph(cfdb_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
}

// Dynamic shared memory of the staged kernel: `slots` slots of 4 field
// tiles, each the item's C columns plus n rows either side and the alignment
// slack.
int ring_cap(int threads, int nmax) { return (threads + 2 * nmax + 8 + 3) / 4 * 4; }
size_t ring_smem(int slots, int threads, int nmax) { return size_t(slots) * 4 * ring_cap(threads, nmax) * sizeof(float); }
constexpr size_t kRingSmemPerSm = 220 * 1024;
// 8 slots where ctas_per_sm CTAs hold them, else 4 (0: not even 4 fit)
int ring_slots(int threads, int ctas_per_sm, int nmax) {
  for (int slots : {8, 4})
    if (ring_smem(slots, threads, nmax) * size_t(ctas_per_sm) <= kRingSmemPerSm) return slots;
  return 0;
}

// The staged kernel runs when both pools start on a 16-byte boundary and its
// ring fits the shared memory of ctas_per_sm CTAs on one SM; otherwise the
// column march (same arithmetic, same results) runs.
bool ring_ok(const cfdb_batch* b, int threads, int ctas_per_sm, const void* a, const void* out) {
  if ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(out)) & 15u) return false;
  return ring_slots(threads, ctas_per_sm, b->nmax) > 0 && (threads + 32) * ctas_per_sm <= 2048;
}

int launch(cfdb_batch* b, const void* a, void* out) {
  const int grid = std::max(1, b->ctx->num_sms) * b->ctas_per_sm;
  if (b->staged == kFormRing && ring_ok(b, b->threads, b->ctas_per_sm, a, out)) {
    const int slots = ring_slots(b->threads, b->ctas_per_sm, b->nmax);
    const size_t smem = ring_smem(slots, b->threads, b->nmax);
    auto kern = slots == 8 ? batch_ring_k<8> : batch_ring_k<4>;
    static size_t attr_set[2][kMaxDevices] = {};
    const int dev = b->ctx->device;
    if (dev < 0 || dev >= kMaxDevices) return cfdb_fail(b->ctx, CFDB_EUNSUPPORTED, "device ordinal %d", dev);
    if (attr_set[slots == 8][dev] < smem) {
      CFDB_CUDA(b->ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
      attr_set[slots == 8][dev] = smem;
    }
    // a persistent grid must be resident at once: clamp to the occupancy
    const int64_t key = int64_t(b->threads) << 32 | int64_t(smem) << 1 | (slots == 8);
    if (b->ring_resident_key != key) {
      int res = 0;
      CFDB_CUDA(b->ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&res, kern, b->threads + 32, smem));
      b->ring_resident = std::max(1, res);
      b->ring_resident_key = key;
    }
    const int rgrid = std::max(1, b->ctx->num_sms) * std::min(b->ctas_per_sm, b->ring_resident);
    RingArgs A{b->threads, ring_cap(b->threads, b->nmax), b->ctx->wait_cycles};
    kern<<<rgrid, b->threads + 32, smem, b->ctx->stream>>>(b->d_probs, b->d_items, b->n_items,
                                                           static_cast<const float*>(a), static_cast<float*>(out), A,
                                                           b->ctx->d_error);
  } else if (b->staged == kFormMarch48 && b->threads <= 256) {
    batch_step_k<256, 5><<<grid, b->threads, 0, b->ctx->stream>>>(b->d_probs, b->d_items, b->n_items,
                                                                   static_cast<const float*>(a), static_cast<float*>(out),
                                                                   b->heat_cols);
  } else {
    batch_step_k<1024, 1><<<grid, b->threads, 0, b->ctx->stream>>>(b->d_probs, b->d_items, b->n_items,
                                                                    static_cast<const float*>(a), static_cast<float*>(out),
                                                                    b->heat_cols);
  }
  CFDB_LAUNCHED(b->ctx);
  return CFDB_OK;
}

std::string cache_key(const cfdb_batch* b) {
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, b->ctx->device);
  uint64_t h = 1469598103934665603ull;  // FNV-1a over (n, kind) of every problem
  for (const auto& p : b->probs) {
    for (int32_t v : {p.n, p.kind}) {
      for (int k = 0; k < 4; ++k) {
        h ^= uint64_t((v >> (8 * k)) & 0xff);
        h *= 1099511628211ull;
      }
    }
  }
  char buf[256];
  std::string name(prop.name);
  for (auto& ch : name)
    if (ch == '"' || ch == ' ') ch = '_';
  // "forms": entries of this kernel generation hold the winning form too;
  // entries tuned for an earlier kernel never match
  snprintf(buf, sizeof(buf), "forms2:%s:%d:%016llx", name.c_str(), int(b->probs.size()), (unsigned long long)h);
  return buf;
}

// The cache file is a flat JSON object
// {"key": [cells_per_item, threads, ctas_per_sm, staged], ...}.
std::map<std::string, std::vector<int>> read_cache(const char* path) {
  std::map<std::string, std::vector<int>> out;
  if (!path) return out;
  std::ifstream f(path);
  if (!f) return out;
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string s = ss.str();
  size_t pos = 0;
  while ((pos = s.find('"', pos)) != std::string::npos) {
    const size_t end = s.find('"', pos + 1);
    if (end == std::string::npos) break;
    const std::string key = s.substr(pos + 1, end - pos - 1);
    const size_t lb = s.find('[', end), rb = s.find(']', end);
    if (lb == std::string::npos || rb == std::string::npos) break;
    int v0 = 0, v1 = 0, v2 = 0, v3 = 0;
    if (sscanf(s.c_str() + lb, "[%d , %d , %d , %d]", &v0, &v1, &v2, &v3) == 4) out[key] = {v0, v1, v2, v3};
    pos = rb + 1;
  }
  return out;
}

// Written to a temporary file and renamed into place, so processes tuning
// at the same time (one per GPU) never leave a torn cache for each other.
void write_cache(const char* path, const std::map<std::string, std::vector<int>>& m) {
  if (!path) return;
  const std::string tmp = std::string(path) + ".tmp" + std::to_string(long(getpid()));
  {
    std::ofstream f(tmp);
    if (!f) return;
    f << "{\n";
    size_t k = 0;
    for (const auto& kv : m) {
      f << "  \"" << kv.first << "\": [" << kv.second[0] << ", " << kv.second[1] << ", " << kv.second[2] << ", "
        << kv.second[3] << "]" << (++k < m.size() ? ",\n" : "\n");
    }
    f << "}\n";
    if (!f) {
      std::remove(tmp.c_str());
      return;
    }
  }
  if (std::rename(tmp.c_str(), path) != 0) std::remove(tmp.c_str());
}

}  // namespace

extern "C" int cfdb_batch_create(cfdb_ctx* ctx, cfdb_problem* probs, int32_t count, int64_t* pool_elems,
                                 cfdb_batch** out) {
  if (!out) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_batch_create: out is NULL");
  *out = nullptr;
  if (!ctx || !probs || count < 1) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_batch_create: need a context and >= 1 problem");
  int64_t off = kPoolPad;  // the column march reads one float before a column's first cell
  for (int32_t i = 0; i < count; ++i) {
    cfdb_problem& p = probs[i];
    if (p.n < 2 || p.n > 1024) return cfdb_fail(ctx, CFDB_EINVAL, "problem %d: n = %d outside [2, 1024]", i, p.n);
    if (p.kind != 0 && p.kind != 1) return cfdb_fail(ctx, CFDB_EINVAL, "problem %d: kind %d is not 0 (heat) or 1 (wave)", i, p.kind);
    if (!(p.param > 0) || !(p.dt > 0) || !std::isfinite(p.param) || !std::isfinite(p.dt))
      return cfdb_fail(ctx, CFDB_EINVAL, "problem %d: param and dt must be finite and > 0", i);
    p.offset = off;
    off += int64_t(p.n) * p.n * p.n * (p.kind == 1 ? 4 : 1);
  }
  const int64_t cells = off;
  off += kPoolPad;  // the staged kernel's copies end on a 16-byte boundary; the march reads one past
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  auto* b = new (std::nothrow) cfdb_batch();
  if (!b) return cfdb_fail(ctx, CFDB_ENOMEM, "host allocation failed");
  b->ctx = ctx;
  b->probs.assign(probs, probs + count);
  b->pool = off;
  for (int32_t i = 0; i < count; ++i) b->nmax = std::max(b->nmax, probs[i].n);
  (void)cells;
  std::vector<ProbDev> pd(count);
  for (int32_t i = 0; i < count; ++i) {
    const cfdb_problem& p = probs[i];
    const double dx = 1.0 / p.n;
    ProbDev d{p.n, p.kind, 0.f, 0.f, 0.f, p.offset};
    if (p.kind == 0) {
      d.c0 = float(p.dt * p.param / (dx * dx));
    } else {
      d.c0 = float(0.5 * p.dt * p.param * p.param / dx);
      d.c1 = float(0.5 * p.dt * p.param / dx);
      d.c2 = float(0.5 * p.dt / dx);
    }
    pd[i] = d;
  }
  int rc = cfdb_dev_alloc(ctx, int64_t(sizeof(ProbDev)) * count, reinterpret_cast<void**>(&b->d_probs));
  if (!rc) {
    cudaError_t e = cudaMemcpy(b->d_probs, pd.data(), sizeof(ProbDev) * count, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) rc = cfdb_cuda_fail(ctx, e, "cudaMemcpy");
  }
  if (!rc) rc = build_items(b);
  if (rc) {
    cfdb_batch_destroy(b);
    return rc;
  }
  if (pool_elems) *pool_elems = off;
  cfdb_adopt(ctx, b, [b] {
    drop_graph(b);
    b->ctx = nullptr;
    b->d_probs = nullptr;
    b->d_items = nullptr;
  });
  *out = b;
  return CFDB_OK;
}

extern "C" int cfdb_batch_destroy(cfdb_batch* b) {
  if (!b) return CFDB_OK;
  drop_graph(b);
  if (b->ctx) {
    cfdb_release(b->ctx, b);
    cudaStreamSynchronize(b->ctx->stream);
    cfdb_dev_free(b->ctx, b->d_probs);
    cfdb_dev_free(b->ctx, b->d_items);
  }
  delete b;
  return CFDB_OK;
}

extern "C" int cfdb_batch_set_config(cfdb_batch* b, int32_t cells_per_item, int32_t threads, int32_t ctas_per_sm) {
  if (!b || !b->ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_batch_set_config: handle is NULL or its context was destroyed");
  if (cells_per_item < 32 || cells_per_item > (1 << 22) || threads < 32 || threads > 1024 || threads % 32 ||
      ctas_per_sm < 1 || ctas_per_sm > 32 || threads * ctas_per_sm > 2048)
    return cfdb_fail(b->ctx, CFDB_EINVAL, "cfdb_batch_set_config: configuration out of range");
  const bool items_change = cells_per_item != b->cells_per_item || threads != b->threads;
  b->cells_per_item = cells_per_item;
  b->threads = threads;
  b->ctas_per_sm = ctas_per_sm;
  drop_graph(b);
  return items_change ? build_items(b) : CFDB_OK;
}

extern "C" int cfdb_batch_set_staged(cfdb_batch* b, int staged) {
  if (!b || !b->ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_batch_set_staged: handle is NULL or its context was destroyed");
  if (staged < kFormMarch || staged > kFormMarch48)
    return cfdb_fail(b->ctx, CFDB_EINVAL, "cfdb_batch_set_staged: form %d is not 0, 1 or 2", staged);
  const bool items_change = (staged == kFormRing) != (b->staged == kFormRing);  // heat item width differs
  b->staged = staged;
  drop_graph(b);
  return items_change ? build_items(b) : CFDB_OK;
}

extern "C" int cfdb_batch_get_config(const cfdb_batch* b, int32_t* cells_per_item, int32_t* threads, int32_t* ctas) {
  if (!b || !b->ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_batch_get_config: handle is NULL or its context was destroyed");
  if (cells_per_item) *cells_per_item = b->cells_per_item;
  if (threads) *threads = b->threads;
  if (ctas) *ctas = b->ctas_per_sm;
  return CFDB_OK;
}

extern "C" int cfdb_batch_step(cfdb_batch* b, const void* a, void* out) {
  if (!b || !b->ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_batch_step: handle is NULL or its context was destroyed");
  if (!a || !out || a == out) return cfdb_fail(b->ctx, CFDB_EINVAL, "cfdb_batch_step: need distinct pools");
  CFDB_CUDA(b->ctx, cudaSetDevice(b->ctx->device));
  return launch(b, a, out);
}

extern "C" int cfdb_batch_run(cfdb_batch* b, void* a, void* out, int32_t steps, int use_graph) {
  CfdbRange range_("cfdb_batch_run");
  if (!b || !b->ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_batch_run: handle is NULL or its context was destroyed");
  if (!a || !out || a == out || steps < 0) return cfdb_fail(b->ctx, CFDB_EINVAL, "cfdb_batch_run: bad arguments");
  CFDB_CUDA(b->ctx, cudaSetDevice(b->ctx->device));
  b->last_launches = 0;
  if (!use_graph) {
    for (int32_t k = 0; k < steps; ++k) {
      if (int rc = (k & 1) ? launch(b, out, a) : launch(b, a, out)) return rc;
      ++b->last_launches;
    }
    return CFDB_OK;
  }
  // (re)record the two-step graph a -> out -> a when pools or config changed
  if (!b->graph || b->graph_a != a || b->graph_b != out || b->graph_cfg[0] != b->cells_per_item ||
      b->graph_cfg[1] != b->threads || b->graph_cfg[2] != b->ctas_per_sm) {
    drop_graph(b);
    cfdb_ctx* ctx = b->ctx;
    if (!ctx->capture_stream)
      CFDB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->capture_stream, cudaStreamNonBlocking));
    cudaStream_t user = ctx->stream;
    ctx->stream = ctx->capture_stream;
    cudaGraph_t g = nullptr;
    int rc = CFDB_OK;
    const int64_t before = ctx->launches;  // recorded launches run only when replayed
    cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      rc = launch(b, a, out);
      if (!rc) rc = launch(b, out, a);
      cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &g);
      if (!rc && e2 != cudaSuccess) rc = cfdb_cuda_fail(ctx, e2, "cudaStreamEndCapture");
    } else {
      rc = cfdb_cuda_fail(ctx, e, "cudaStreamBeginCapture");
    }
    ctx->launches = before;
    ctx->stream = user;
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      b->graph = nullptr;
      return cfdb_cuda_fail(ctx, e, "cudaGraphInstantiate");
    }
    b->graph_a = a;
    b->graph_b = out;
    b->graph_cfg[0] = b->cells_per_item; b->graph_cfg[1] = b->threads; b->graph_cfg[2] = b->ctas_per_sm;
  }
  for (int32_t k = 0; k + 1 < steps; k += 2) {
    CFDB_CUDA(b->ctx, cudaGraphLaunch(b->graph, b->ctx->stream));
    b->last_launches += 2;
    b->ctx->launches += 2;
  }
  if (steps & 1) {
    if (int rc = launch(b, a, out)) return rc;
    ++b->last_launches;
  }
  return CFDB_OK;
}

extern "C" int cfdb_batch_launch_count(const cfdb_batch* b, int64_t* out) {
  if (!b || !out) return cfdb_fail(b ? b->ctx : nullptr, CFDB_EINVAL, "cfdb_batch_launch_count: bad arguments");
  *out = b->last_launches;
  return CFDB_OK;
}

extern "C" int cfdb_batch_tune(cfdb_batch* b, void* a, void* out, const char* cache_path) {
  if (!b || !b->ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_batch_tune: handle is NULL or its context was destroyed");
  if (!a || !out || a == out) return cfdb_fail(b->ctx, CFDB_EINVAL, "cfdb_batch_tune: need distinct pools");
  cfdb_ctx* ctx = b->ctx;
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  auto cache = read_cache(cache_path);
  const std::string key = cache_key(b);
  auto hit = cache.find(key);
  if (hit != cache.end() && hit->second.size() == 4) {
    if (cfdb_batch_set_staged(b, std::min(std::max(hit->second[3], kFormMarch), kFormMarch48)) == CFDB_OK &&
        cfdb_batch_set_config(b, hit->second[0], hit->second[1], hit->second[2]) == CFDB_OK)
      return CFDB_OK;
  }
  cudaEvent_t e0, e1;
  CFDB_CUDA(ctx, cudaEventCreate(&e0));
  CFDB_CUDA(ctx, cudaEventCreate(&e1));
  float best = INFINITY;
  int bc[4] = {b->cells_per_item, b->threads, b->ctas_per_sm, b->staged};
  int rc = CFDB_OK;
  // Both kernel forms.  The column march times items of 512-8192 cells at
  // 2-16 CTAs per SM; the staged kernel keeps several planes in flight per
  // CTA, so it wants longer items and fewer, larger CTAs (shared memory
  // bounds them), and only configurations it takes are timed.
  for (int form : {kFormMarch, kFormMarch48, kFormRing}) {
    if ((rc = cfdb_batch_set_staged(b, form))) break;
    const bool ring = form == kFormRing;
    const std::vector<int> cpis = ring ? std::vector<int>{2048, 8192, 32768, 131072}
                                       : std::vector<int>{512, 1024, 2048, 4096, 8192};
    const std::vector<int> ths = form == kFormMarch48 ? std::vector<int>{128, 256} : std::vector<int>{128, 256, 512};
    const std::vector<int> ctas = ring ? std::vector<int>{1, 2, 3, 4}
                                       : (form == kFormMarch48 ? std::vector<int>{5, 10} : std::vector<int>{2, 4, 8, 16});
    for (int cpi : cpis)
      for (int th : ths)
        for (int ct : ctas) {
          if (th * ct > 2048 || rc) continue;
          if (ring && !ring_ok(b, th, ct, a, out)) continue;
          if ((rc = cfdb_batch_set_config(b, cpi, th, ct))) break;
          if ((rc = launch(b, a, out))) break;  // warm-up
          cudaEventRecord(e0, ctx->stream);
          for (int k = 0; k < 4 && !rc; ++k) rc = (k & 1) ? launch(b, out, a) : launch(b, a, out);
          cudaEventRecord(e1, ctx->stream);
          cudaError_t e = cudaEventSynchronize(e1);
          if (e != cudaSuccess) rc = cfdb_cuda_fail(ctx, e, "cudaEventSynchronize");
          if (rc) break;
          float ms = 0;
          cudaEventElapsedTime(&ms, e0, e1);
          if (ms < best) {
            best = ms;
            bc[0] = cpi; bc[1] = th; bc[2] = ct; bc[3] = form;
          }
        }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!rc) rc = cfdb_check_device_error(ctx);  // a staged candidate whose wait ran out
  if (rc) return rc;
  if ((rc = cfdb_batch_set_staged(b, bc[3]))) return rc;
  if ((rc = cfdb_batch_set_config(b, bc[0], bc[1], bc[2]))) return rc;
  cache[key] = {bc[0], bc[1], bc[2], bc[3]};
  write_cache(cache_path, cache);
  return CFDB_OK;
}
