// TMA-staged 7-point stencil sweep for uniform hexahedral meshes (sm_100a).
//
// One CTA owns a TZ x TY column of cells in the (z, y) plane and marches a
// chunk of x planes.  For every plane a single 4-D TMA load
// (cp.async.bulk.tensor.4d, no cluster multicast) brings all NF fields of the
// (TZ+8) x (TY+2) tile -- the tile plus its one-cell y halo and a z halo
// widened to 4 cells so the innermost coordinate stays 16-byte aligned --
// into a ring of S shared-memory slots guarded by mbarriers.  Each thread
// owns 4 consecutive z cells (one float4 per field): the x neighbours come
// from registers (the previous and next planes), the y and z neighbours from
// the staged tile.  Out-of-domain neighbours are replaced by the physics'
// ghost state (zero-gradient or reflective), so the TMA zero fill outside the
// domain is never read.
//
// Requirements checked by the host: nz % 4 == 0 (16-byte row strides and
// aligned z origins), float32 state stored field after field.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace stencil {

// ---- PTX wrappers ------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Brings a tensor map (a __grid_constant__ kernel parameter) into the TMA
// unit's descriptor cache ahead of its first copy.
__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* m) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(m)) : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// try_wait with a suspend-time hint: a thread whose phase is not complete yet
// may sleep up to `ns` nanoseconds (woken early when the phase completes)
// instead of returning at once, so waiting warps leave the issue slots to
// others.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, uint32_t parity, uint32_t ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

// Programmatic dependent launch: the sweep is launched with programmatic
// stream serialisation, so its CTAs may become resident while the previous
// kernel of the stream drains.  grid_dep_wait() blocks until that kernel has
// completed and its writes are visible; it precedes every global-memory access
// of the sweep (reads AND writes: the next step writes the buffer the previous
// one reads).  grid_dep_launch() lets the next kernel start its own prologue.
// Both are no-ops when the launch carries no programmatic dependency.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Bounded wait: gives up after `limit` SM clock cycles (default ~2 s) so a
// lost transaction can never hang the GPU; the caller records the failure in
// the error word.
constexpr long long kWaitCycles = 4000000000LL;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long limit) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > limit) return false;
  return true;
}

// The same bound with sleeping polls (mbar_try_wait_sleep).
__device__ __forceinline__ bool mbar_wait_bounded_sleep(uint64_t* bar, uint32_t parity, long long limit) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait_sleep(bar, parity, 20000u))
    if (clock64() - t0 > limit) return false;
  return true;
}

// Device error word codes (ctx->d_error[0]).
constexpr int kErrWaitTimeout = 1;
constexpr int kErrSmemAlign = 2;
constexpr int kErrSmemSize = 3;

// ---- the sweep -------------------------------------------------------------
struct Geometry {
  int X, Y, Z;      // cells
  int chunks;       // x chunks; chunk c covers planes [c X / chunks, (c+1) X / chunks)
  long long n;      // X*Y*Z
  long long wait_cycles;  // bound of every mbarrier wait, SM clock cycles
  // Test hook (-1: off): CTA (0, 0) arms the barrier of its plane k ==
  // missing_plane with the plane's byte count but issues no copy for it, so
  // the wait on that plane runs out (the timeout path, without a fault).
  int missing_plane;
};

// Staged fields of one cell and its six neighbours (x-, x+, y-, y+, z-, z+).
// The FT staged fields are the NF state fields (read from `q`, written to
// `out`), then NA auxiliary fields (read from `aux`), then the coefficient
// field c when HAS_C.  Neighbours beyond a wall hold Phys::ghost(P, dir);
// bit 2*dir + side of `walls` marks them.  (Conservative schemes that
// evaluate each face once run on the face sweep, face_sweep.cuh.)
template <int FT> struct CellIn {
  float P[FT];
  float nb[6][FT];
  int walls;
  long long idx;  // cell id
  float pre;      // Phys::pre_ptr(params)[idx], loaded one plane ahead (physics with HAS_PRE)
};

// Physics that read one per-cell value from global memory besides the staged
// fields (Phys::HAS_PRE, pointer Phys::pre_ptr(params)): the sweep loads the
// next plane's values while the current plane is computed, so the load
// latency hides behind a plane of work.
template <class P, class = void> struct has_pre { static constexpr bool value = false; };
template <class P> struct has_pre<P, decltype(void(P::HAS_PRE))> { static constexpr bool value = P::HAS_PRE; };

// Paired physics (Phys::PAIRED): with two cells per thread (VZ == 2) the sweep
// calls Phys::cell2(in0, in1, params, o0, o1) once instead of cell() twice, so
// the physics can advance both cells with packed FP32 pairs (f32x2.cuh).
template <class P, class = void> struct is_paired { static constexpr bool value = false; };
template <class P> struct is_paired<P, decltype(void(P::PAIRED))> { static constexpr bool value = P::PAIRED; };

// Phys provides:
//   static constexpr int NF, NA;        state fields (read and written), auxiliary fields (read)
//   static constexpr bool HAS_C;        a per-cell coefficient field is staged as the last field
//   static constexpr int MIN_BLOCKS;    resident CTAs per SM the register budget must allow
//   struct Params;                      kernel parameters (by value)
//   struct Acc;                         per-thread epilogue accumulator
//   __device__ static bool begin(Params&)  -> false: skip the sweep (e.g. a finished clock); may
//        fill per-launch values (a device-side dt) into its copy of the parameters
//   __device__ static void ghost(float g[FT], const float p[FT], int dir);   dir 0=x,1=y,2=z
//   __device__ static void cell(const CellIn<FT>&, const Params&, float out[NF]);
//   __device__ static void acc_init(Acc&), acc_cell(Acc&, const float out[NF], const Params&)
//   __device__ static void finish(Acc&, const Params&, bool thread_active)   (called by all threads)
template <int TZ, int TY, int S, int NF, int NA, bool HAS_C, int VZ> struct Layout {
  static constexpr int FT = NF + NA + (HAS_C ? 1 : 0);  // staged fields
  static constexpr int RL = TZ + 8;                       // row length (floats)
  static constexpr int RR = TY + 2;                       // rows
  static constexpr int TILE = RL * RR;                    // floats per field tile
  static constexpr int A_OFF = (NF * TILE + 31) / 32 * 32;              // 128-byte aligned
  static constexpr int C_OFF = (A_OFF + NA * TILE + 31) / 32 * 32;      // 128-byte aligned
  static constexpr int SLOT = (C_OFF + (HAS_C ? TILE : 0) + 31) / 32 * 32;
  static constexpr uint32_t TX_BYTES = uint32_t(4 * TILE * FT);
  static constexpr size_t SMEM_BYTES = size_t(S) * SLOT * 4;
  static constexpr int THREADS = (TZ / VZ) * TY;
  __host__ __device__ static constexpr int off(int f) {
    return f < NF ? f * TILE : (f < NF + NA ? A_OFF + (f - NF) * TILE : C_OFF);
  }
};

template <int VZ> __device__ __forceinline__ void ldv(const float* p, float* v) {
  if constexpr (VZ == 4) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  } else if constexpr (VZ == 2) {
    const float2 t = *reinterpret_cast<const float2*>(p);
    v[0] = t.x; v[1] = t.y;
  } else {
    v[0] = *p;
  }
}

template <int VZ> __device__ __forceinline__ void stv(float* p, const float* v) {
  if constexpr (VZ == 4) *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  else if constexpr (VZ == 2) *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
  else *p = v[0];
}

template <class Phys, int TZ, int TY, int S, int VZ>
__global__ void __launch_bounds__((TZ / VZ) * TY, Phys::MIN_BLOCKS)
    sweep_kernel(const __grid_constant__ CUtensorMap tm_q, const __grid_constant__ CUtensorMap tm_a,
                 const __grid_constant__ CUtensorMap tm_c, Geometry g, float* __restrict__ out,
                 typename Phys::Params prm, int* __restrict__ err) {
  constexpr int NF = Phys::NF;
  constexpr int NA = Phys::NA;
  constexpr bool PRE = has_pre<Phys>::value;
  constexpr bool PAIR = is_paired<Phys>::value && VZ == 2;
  using L = Layout<TZ, TY, S, NF, NA, Phys::HAS_C, VZ>;
  constexpr int FT = L::FT;
  // Indexing the extern array directly keeps the accesses in the shared
  // address space (LDS, not generic loads); its start must be 128-byte aligned
  // for TMA, which is checked before the first copy is issued.
  extern __shared__ __align__(128) float smem[];
  __shared__ __align__(8) uint64_t bars[S];
  // Issuer bookkeeping in shared memory (thread 0 only), so it holds no
  // register through the plane loop: the last plane whose copies were
  // issued, and, once a wait gave up, the copies to drain (bit s: slot s
  // holds an issued copy not waited on yet; bit 16 + s: its parity).
  static_assert(S <= 16, "the drain word holds 16 slots");
  __shared__ int last_issued;
  __shared__ uint32_t drain;

  const int ntz = (g.Z + TZ - 1) / TZ;
  const int z0 = (blockIdx.x % ntz) * TZ;
  const int y0 = (blockIdx.x / ntz) * TY;
  const int x0 = int((long long)blockIdx.y * g.X / g.chunks);
  const int x1 = int((long long)(blockIdx.y + 1) * g.X / g.chunks);
  if (x0 >= x1) return;
  // Set-up that touches no global memory runs before the wait for the
  // previous kernel, overlapping its last CTAs: the ring's barriers and the
  // tensor maps' descriptors.
  if (threadIdx.x == 0) {
    prefetch_tmap(&tm_q);
    if constexpr (NA > 0) prefetch_tmap(&tm_a);
    if constexpr (Phys::HAS_C) prefetch_tmap(&tm_c);
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
    last_issued = -1;
    drain = 0;
  }
  __syncthreads();
  grid_dep_wait();
  grid_dep_launch();
  if (smem_u32(smem) & 127u) {
    if (threadIdx.x == 0) atomicExch(err, kErrSmemAlign);
    return;
  }
  {
    // the launch must provide the layout's dynamic shared memory (the ring)
    uint32_t dyn;
    asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    if (dyn < L::SMEM_BYTES) {
      if (threadIdx.x == 0) atomicExch(err, kErrSmemSize);
      return;
    }
  }
  typename Phys::Params P = prm;
  if (!Phys::begin(P)) return;

  const int tz = threadIdx.x % (TZ / VZ);
  const int ty = threadIdx.x / (TZ / VZ);
  const int y = y0 + ty;
  const int zb = z0 + VZ * tz;
  const bool active = (y < g.Y) && (zb < g.Z);
  const int kmax = x1 - x0 + 1;  // plane k <-> x = x0 - 1 + k

  // A wait that gives up (bad) ends the staging: the issuing thread (0)
  // issues nothing more and lets the copies it already issued land before
  // the CTA can exit, every later wait is skipped, and the error word
  // reports the timeout.  The results of such a launch are invalid.
  bool bad = false;
  auto issue = [&](int k) {
    const int x = x0 - 1 + k;
    if (bad || k > kmax || x < 0 || x >= g.X) return;
    const int s = k % S;
    float* dst = smem + s * L::SLOT;
    mbar_expect_tx(&bars[s], L::TX_BYTES);
    last_issued = k;
    if (k == g.missing_plane && blockIdx.x == 0 && blockIdx.y == 0) return;
    tma_load_4d(dst, &tm_q, z0 - 4, y0 - 1, x, 0, &bars[s]);
    if constexpr (NA > 0) tma_load_4d(dst + L::A_OFF, &tm_a, z0 - 4, y0 - 1, x, 0, &bars[s]);
    if constexpr (Phys::HAS_C) tma_load_3d(dst + L::C_OFF, &tm_c, z0 - 4, y0 - 1, x, &bars[s]);
  };
  if (threadIdx.x == 0)
    for (int k = 0; k < S; ++k) issue(k);

  uint32_t parity = 0;  // bit s: parity of the next completion of slot s
  auto wait_plane = [&](int k) {
    const int s = k % S;
    const uint32_t par = (parity >> s) & 1u;
    parity ^= 1u << s;
    if (bad) return;
    if (!mbar_wait_bounded(&bars[s], par, g.wait_cycles)) {
      bad = true;
      // planes k+1 .. last_issued sit in other slots, none waited on yet:
      // their bits in `parity` are the parities of those copies' completions
      if (threadIdx.x == 0) {
        uint32_t d = (parity & 0xffffu) << 16;
        for (int j = k + 1; j <= last_issued; ++j) d |= 1u << (j % S);
        drain = d;
      }
    }
  };
  const int ctr = (ty + 1) * L::RL + 4 + VZ * tz;  // thread's first cell in a field tile
  auto load_center = [&](int k, float v[FT][VZ]) {
    const float* base = smem + (k % S) * L::SLOT;
#pragma unroll
    for (int f = 0; f < FT; ++f) ldv<VZ>(base + L::off(f) + ctr, v[f]);
  };
  auto ghostv = [&](float dst[FT][VZ], const float src[FT][VZ], int dir) {
#pragma unroll
    for (int j = 0; j < VZ; ++j) {
      float a[FT], b[FT];
#pragma unroll
      for (int f = 0; f < FT; ++f) a[f] = src[f][j];
      Phys::ghost(b, a, dir);
#pragma unroll
      for (int f = 0; f < FT; ++f) dst[f][j] = b[f];
    }
  };

  float prv[FT][VZ], cur[FT][VZ], nxt[FT][VZ];
  if (x0 > 0) {
    wait_plane(0);
    load_center(0, prv);
  }
  wait_plane(1);
  load_center(1, cur);
  if (x0 == 0) ghostv(prv, cur, 0);
  __syncthreads();
  if (threadIdx.x == 0) {
    fence_proxy_async();
    issue(S);
  }

  typename Phys::Acc acc;
  Phys::acc_init(acc);
  const long long plane = (long long)g.Y * g.Z;
  const int wy = (y == 0 ? 4 : 0) | (y == g.Y - 1 ? 8 : 0);
  // HAS_PRE: the per-cell global value of the current plane (preC) and the next one (preN)
  float preC[VZ], preN[VZ];
  const long long col = (long long)y * g.Z + zb;
  if constexpr (PRE) {
    if (active) ldv<VZ>(Phys::pre_ptr(P) + ((long long)x0 * plane + col), preC);
  }

  for (int x = x0; x < x1; ++x) {
    const int k = x - x0 + 1;
    if constexpr (PRE) {
      if (active && x + 1 < x1) ldv<VZ>(Phys::pre_ptr(P) + ((long long)(x + 1) * plane + col), preN);
    }
    if (x + 1 < g.X) {
      wait_plane(k + 1);
      load_center(k + 1, nxt);
    } else {
      ghostv(nxt, cur, 0);
    }
    if (active) {
      const float* base = smem + (k % S) * L::SLOT;
      float ym[FT][VZ], yp[FT][VZ], zl[FT], zr[FT];
#pragma unroll
      for (int f = 0; f < FT; ++f) {
        const float* t = base + L::off(f);
        ldv<VZ>(t + ctr - L::RL, ym[f]);
        ldv<VZ>(t + ctr + L::RL, yp[f]);
        zl[f] = t[ctr - 1];
        zr[f] = t[ctr + VZ];
      }
      if (wy & 4) ghostv(ym, cur, 1);
      if (wy & 8) ghostv(yp, cur, 1);
      const int wx = (x == 0 ? 1 : 0) | (x == g.X - 1 ? 2 : 0);
      float res[NF][VZ];
      CellIn<FT> ins[VZ];
#pragma unroll
      for (int j = 0; j < VZ; ++j) {
        CellIn<FT>& in = ins[j];
#pragma unroll
        for (int f = 0; f < FT; ++f) {
          in.P[f] = cur[f][j];
          in.nb[0][f] = prv[f][j];
          in.nb[1][f] = nxt[f][j];
          in.nb[2][f] = ym[f][j];
          in.nb[3][f] = yp[f][j];
          in.nb[4][f] = j == 0 ? zl[f] : cur[f][j - 1];
          in.nb[5][f] = j == VZ - 1 ? zr[f] : cur[f][j + 1];
        }
        int w = wx | wy;
        if (j == 0 && zb == 0) {
          Phys::ghost(in.nb[4], in.P, 2);
          w |= 16;
        }
        if (j == VZ - 1 && zb + VZ - 1 == g.Z - 1) {
          Phys::ghost(in.nb[5], in.P, 2);
          w |= 32;
        }
        in.walls = w;
        in.idx = (long long)x * plane + (long long)y * g.Z + zb + j;
        if constexpr (PRE) in.pre = preC[j];
        if constexpr (!PAIR) {
          float o[NF];
          Phys::cell(in, P, o);
          Phys::acc_cell(acc, o, P);
#pragma unroll
          for (int f = 0; f < NF; ++f) res[f][j] = o[f];
        }
      }
      if constexpr (PAIR) {
        float o0[NF], o1[NF];
        Phys::cell2(ins[0], ins[1], P, o0, o1);
        Phys::acc_cell(acc, o0, P);
        Phys::acc_cell(acc, o1, P);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          res[f][0] = o0[f];
          res[f][1] = o1[f];
        }
      }
      const long long idx = (long long)x * plane + (long long)y * g.Z + zb;
#pragma unroll
      for (int f = 0; f < NF; ++f) stv<VZ>(out + f * g.n + idx, res[f]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      fence_proxy_async();
      issue(k + S);
    }
#pragma unroll
    for (int f = 0; f < FT; ++f)
#pragma unroll
      for (int j = 0; j < VZ; ++j) {
        prv[f][j] = cur[f][j];
        cur[f][j] = nxt[f][j];
      }
    if constexpr (PRE) {
#pragma unroll
      for (int j = 0; j < VZ; ++j) preC[j] = preN[j];
    }
  }
  if (bad) {
    // the copies still in flight land in shared memory before the CTA exits
    if (threadIdx.x == 0)
      for (int t = 0; t < S; ++t)
        if ((drain >> t) & 1u) mbar_wait_bounded(&bars[t], (drain >> (16 + t)) & 1u, g.wait_cycles);
    atomicExch(err, kErrWaitTimeout);
  }
  Phys::finish(acc, P, active);
}

}  // namespace stencil
