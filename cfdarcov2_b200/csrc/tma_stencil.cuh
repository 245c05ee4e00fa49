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

// Bounded wait: gives up after ~2 s of SM clocks so a lost transaction can
// never hang the GPU; the caller records the failure in the error word.
constexpr long long kWaitCycles = 4000000000LL;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > kWaitCycles) return false;
  return true;
}

// Device error word codes (ctx->d_error[0]).
constexpr int kErrWaitTimeout = 1;

// ---- the sweep -------------------------------------------------------------
struct Geometry {
  int X, Y, Z;      // cells
  int chunk;        // x planes per CTA
  long long n;      // X*Y*Z
};

// Phys provides:
//   static constexpr int NF;            fields in the state
//   static constexpr bool HAS_C;        per-cell coefficient field staged too
//   struct Params;                      kernel parameters (by value)
//   struct Acc;                         per-thread epilogue accumulator
//   __device__ static void ghost(float g[NF], const float p[NF], int dir);   dir 0=x,1=y,2=z
//   __device__ static void cell(const float P[NF], const float nb[6][NF], const float cc[7],
//                               const Params&, float out[NF]);
//        nb order: x-, x+, y-, y+, z-, z+; cc: c_P then the 6 neighbours
//   __device__ static void acc_init(Acc&), acc_cell(Acc&, const float out[NF], const Params&)
//   __device__ static void finish(Acc&, const Params&, bool thread_active)   (called by all threads)
//   __device__ static bool begin(Params&)  -> false: skip the sweep (e.g. a finished clock); may
//        fill per-launch values (a device-side dt) into its copy of the parameters
template <int TZ, int TY, int S, int NF, bool HAS_C> struct Layout {
  static constexpr int RL = TZ + 8;                       // row length (floats)
  static constexpr int RR = TY + 2;                       // rows
  static constexpr int TILE = RL * RR;                    // floats per field tile
  static constexpr int C_OFF = (NF * TILE + 31) / 32 * 32;
  static constexpr int SLOT = (C_OFF + (HAS_C ? TILE : 0) + 31) / 32 * 32;  // 128-byte multiple
  static constexpr uint32_t TX_BYTES = uint32_t(4 * (NF * TILE + (HAS_C ? TILE : 0)));
  static constexpr size_t SMEM_BYTES = size_t(S) * SLOT * 4 + 128;
  static constexpr int THREADS = (TZ / 4) * TY;
};

template <class Phys, int TZ, int TY, int S>
__global__ void __launch_bounds__((TZ / 4) * TY)
    sweep_kernel(const __grid_constant__ CUtensorMap tm_q, const __grid_constant__ CUtensorMap tm_c, Geometry g,
                 float* __restrict__ out, typename Phys::Params prm, int* __restrict__ err) {
  constexpr int NF = Phys::NF;
  using L = Layout<TZ, TY, S, NF, Phys::HAS_C>;
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bars[S];
  float* smem = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));

  const int ntz = (g.Z + TZ - 1) / TZ;
  const int z0 = (blockIdx.x % ntz) * TZ;
  const int y0 = (blockIdx.x / ntz) * TY;
  const int x0 = blockIdx.y * g.chunk;
  const int x1 = min(g.X, x0 + g.chunk);
  if (x0 >= x1) return;
  typename Phys::Params P = prm;
  if (!Phys::begin(P)) return;

  const int tz = threadIdx.x % (TZ / 4);
  const int ty = threadIdx.x / (TZ / 4);
  const int y = y0 + ty;
  const int zb = z0 + 4 * tz;
  const bool active = (y < g.Y) && (zb < g.Z);
  const int kmax = x1 - x0 + 1;  // plane k <-> x = x0 - 1 + k

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  auto issue = [&](int k) {
    const int x = x0 - 1 + k;
    if (k > kmax || x < 0 || x >= g.X) return;
    const int s = k % S;
    float* dst = smem + s * L::SLOT;
    mbar_expect_tx(&bars[s], L::TX_BYTES);
    tma_load_4d(dst, &tm_q, z0 - 4, y0 - 1, x, 0, &bars[s]);
    if constexpr (Phys::HAS_C) tma_load_3d(dst + L::C_OFF, &tm_c, z0 - 4, y0 - 1, x, &bars[s]);
  };
  if (threadIdx.x == 0)
    for (int k = 0; k < S; ++k) issue(k);

  uint32_t parity = 0;  // bit s: parity of the next completion of slot s
  bool bad = false;
  auto wait_plane = [&](int k) {
    const int s = k % S;
    if (!mbar_wait_bounded(&bars[s], (parity >> s) & 1u)) bad = true;
    parity ^= 1u << s;
  };
  const int ctr = (ty + 1) * L::RL + 4 + 4 * tz;  // thread's float4 in a field tile
  auto load_center = [&](int k, float v[NF][4], float c4[4]) {
    const float* base = smem + (k % S) * L::SLOT;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      const float4 t = *reinterpret_cast<const float4*>(base + f * L::TILE + ctr);
      v[f][0] = t.x; v[f][1] = t.y; v[f][2] = t.z; v[f][3] = t.w;
    }
    if constexpr (Phys::HAS_C) {
      const float4 t = *reinterpret_cast<const float4*>(base + L::C_OFF + ctr);
      c4[0] = t.x; c4[1] = t.y; c4[2] = t.z; c4[3] = t.w;
    }
  };
  auto ghost4 = [&](float dst[NF][4], const float src[NF][4], int dir) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float a[NF], b[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) a[f] = src[f][j];
      Phys::ghost(b, a, dir);
#pragma unroll
      for (int f = 0; f < NF; ++f) dst[f][j] = b[f];
    }
  };

  float prv[NF][4], cur[NF][4], nxt[NF][4];
  float cprv[4] = {0, 0, 0, 0}, ccur[4] = {0, 0, 0, 0}, cnxt[4] = {0, 0, 0, 0};
  if (x0 > 0) {
    wait_plane(0);
    load_center(0, prv, cprv);
  }
  wait_plane(1);
  load_center(1, cur, ccur);
  if (x0 == 0) {
    ghost4(prv, cur, 0);
#pragma unroll
    for (int j = 0; j < 4; ++j) cprv[j] = ccur[j];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    fence_proxy_async();
    issue(S);
  }

  typename Phys::Acc acc;
  Phys::acc_init(acc);
  const long long plane = (long long)g.Y * g.Z;

  for (int x = x0; x < x1; ++x) {
    const int k = x - x0 + 1;
    if (x + 1 < g.X) {
      wait_plane(k + 1);
      load_center(k + 1, nxt, cnxt);
    } else {
      ghost4(nxt, cur, 0);
#pragma unroll
      for (int j = 0; j < 4; ++j) cnxt[j] = ccur[j];
    }
    if (active) {
      const float* base = smem + (k % S) * L::SLOT;
      float ym[NF][4], yp[NF][4], zl[NF], zr[NF];
      float cym[4], cyp[4], czl = 0.f, czr = 0.f;
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const float* t = base + f * L::TILE;
        const float4 a = *reinterpret_cast<const float4*>(t + ctr - L::RL);
        const float4 b = *reinterpret_cast<const float4*>(t + ctr + L::RL);
        ym[f][0] = a.x; ym[f][1] = a.y; ym[f][2] = a.z; ym[f][3] = a.w;
        yp[f][0] = b.x; yp[f][1] = b.y; yp[f][2] = b.z; yp[f][3] = b.w;
        zl[f] = t[ctr - 1];
        zr[f] = t[ctr + 4];
      }
      if constexpr (Phys::HAS_C) {
        const float* t = base + L::C_OFF;
        const float4 a = *reinterpret_cast<const float4*>(t + ctr - L::RL);
        const float4 b = *reinterpret_cast<const float4*>(t + ctr + L::RL);
        cym[0] = a.x; cym[1] = a.y; cym[2] = a.z; cym[3] = a.w;
        cyp[0] = b.x; cyp[1] = b.y; cyp[2] = b.z; cyp[3] = b.w;
        czl = t[ctr - 1];
        czr = t[ctr + 4];
      }
      if (y == 0) {
        ghost4(ym, cur, 1);
        if constexpr (Phys::HAS_C) for (int j = 0; j < 4; ++j) cym[j] = ccur[j];
      }
      if (y == g.Y - 1) {
        ghost4(yp, cur, 1);
        if constexpr (Phys::HAS_C) for (int j = 0; j < 4; ++j) cyp[j] = ccur[j];
      }
      float res[NF][4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        float Pc[NF], nb[6][NF], cc[7];
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          Pc[f] = cur[f][j];
          nb[0][f] = prv[f][j];
          nb[1][f] = nxt[f][j];
          nb[2][f] = ym[f][j];
          nb[3][f] = yp[f][j];
          nb[4][f] = j == 0 ? zl[f] : cur[f][j - 1];
          nb[5][f] = j == 3 ? zr[f] : cur[f][j + 1];
        }
        if (j == 0 && zb == 0) Phys::ghost(nb[4], Pc, 2);
        if (j == 3 && zb + 3 == g.Z - 1) Phys::ghost(nb[5], Pc, 2);
        if constexpr (Phys::HAS_C) {
          cc[0] = ccur[j];
          cc[1] = cprv[j]; cc[2] = cnxt[j]; cc[3] = cym[j]; cc[4] = cyp[j];
          cc[5] = j == 0 ? (zb == 0 ? ccur[0] : czl) : ccur[j - 1];
          cc[6] = j == 3 ? (zb + 3 == g.Z - 1 ? ccur[3] : czr) : ccur[j + 1];
        } else {
#pragma unroll
          for (int q = 0; q < 7; ++q) cc[q] = 0.f;
        }
        float o[NF];
        Phys::cell(Pc, nb, cc, P, o);
        Phys::acc_cell(acc, o, P);
#pragma unroll
        for (int f = 0; f < NF; ++f) res[f][j] = o[f];
      }
      const long long idx = (long long)x * plane + (long long)y * g.Z + zb;
#pragma unroll
      for (int f = 0; f < NF; ++f)
        *reinterpret_cast<float4*>(out + f * g.n + idx) = make_float4(res[f][0], res[f][1], res[f][2], res[f][3]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      fence_proxy_async();
      issue(k + S);
    }
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        prv[f][j] = cur[f][j];
        cur[f][j] = nxt[f][j];
      }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      cprv[j] = ccur[j];
      ccur[j] = cnxt[j];
    }
  }
  if (bad) atomicExch(err, kErrWaitTimeout);
  Phys::finish(acc, P, active);
}

}  // namespace stencil
