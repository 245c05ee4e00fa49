// Face-flux TMA sweep for conservative schemes (sm_100a).
//
// Same data movement as the stencil sweep (tma_stencil.cuh): one CTA owns a
// TZ x TY column of the (z, y) plane, marches a chunk of x planes, and one
// thread (0) streams every plane through a ring of S shared-memory slots with
// cp.async.bulk.tensor (no cluster multicast), one mbarrier per slot.  What
// differs is the work per plane:
//
//  * every face is evaluated once: the flux through a cell's +x face is kept
//    in registers as the next plane's -x flux, the VZ + 1 z faces of a
//    thread's VZ cells are evaluated once each, and each cell evaluates its
//    two y faces;
//  * besides that x flux only the derived values of the next plane's own
//    cells are carried between planes: the state and the geometry of plane k
//    are read from slot k while plane k is computed (the slot is refilled
//    only after the plane's closing barrier), so the register footprint does
//    not grow with the staged fields;
//  * derived values (ND > 0: per-cell quantities such as 1/rho, p, a) are
//    computed once per cell and plane: a thread derives its cells of plane
//    k + 1 while it computes plane k (it needs them for its +x faces anyway),
//    and publishes them, together with the tile's one-cell halo ring (one
//    halo cell per thread), into one of two shared buffers that the y and z
//    neighbours read after the plane's closing barrier;
//  * per cell geometry (NG > 0) is staged next to the state with a halo on the
//    low side only (one row below, four z cells before): a face's geometry is
//    that of the cell on its minus side, so only the -y and -z neighbours'
//    face values are ever needed.  The geometry lives on a lattice padded by
//    one ghost layer below x and y and four cells below z (entry of cell
//    (x, y, z): ((x + 1) Yp + y + 1) Zp + z + 4), whose ghost entries carry
//    the geometry of the -wall faces, so a wall face gets its geometry from
//    the same staged tile as an interior face;
//  * a face on the domain boundary is evaluated between the cell and its
//    ghost (Phys::ghost, built from the cell and the face's geometry), either
//    behind a branch or, for physics whose ghost is a few selects
//    (Phys::SELECT_WALLS), by building the ghost for every boundary-capable
//    face and selecting it, so the flux code is not duplicated per branch.
//
// Phys provides
//   static constexpr int NF;        state fields (read from q, written to out)
//   static constexpr int NG;        geometry fields per cell (read from the padded geometry)
//   static constexpr int NGF;       geometry values per face: the face with normal e_d between L and R
//                                   uses L's fields [d NGF, (d + 1) NGF)
//   static constexpr int ND;        derived values per cell
//   static constexpr bool SELECT_WALLS;
//   static constexpr int MIN_BLOCKS;
//   struct Params; struct Acc;
//   __device__ static bool begin(Params&);
//   __device__ static void derive(const float q[NF], float d[ND], const Params&);   (ND > 0 only)
//   __device__ static void ghost(const float C[NF], const float Cd[ND], const float Sf[NGF], int d,
//                                float g[NF], float gd[ND]);                 the cell beyond a wall face
//   __device__ static void flux(const float L[NF], const float Ld[ND], const float R[NF], const float Rd[ND],
//                               const float Sf[NGF], int d, const Params&, float F[NF]);   along +e_d, L -> R
//   __device__ static void update(const float C[NF], const float Cd[ND], const float G[NG],
//                                 const float dF[3][NF], const Params&, float out[NF]);  dF[d] = F(d+) - F(d-)
//   __device__ static void acc_init(Acc&), acc_cell(Acc&, const float out[NF], const Params&),
//                          finish(Acc&, const Params&, bool thread_active);
//   optionally __device__ static void prologue(const Params&), called by every thread once the
//   first planes' copies are issued (work that needs no plane, hidden behind their latency);
// (array extents of size 0 are passed as 1), and optionally, with two cells
// per thread (VZ == 2), the same operations on (cell 0, cell 1) pairs
// (Phys::PAIRED; derived values, no per-cell geometry), which the physics
// can run as packed f32x2 instructions (the kernel then keeps a thread's
// cells in register pairs throughout; update and acc_cell are needed only in
// pair form):
//   derive2(const float2 q[NF], float2 d[ND], P), flux2(const float2 L[NF], const float2 Ld[ND],
//   const float2 R[NF], const float2 Rd[ND], int d, P, float2 F[NF]), update2(const float2 C[NF],
//   const float2 Cd[ND], const float2 dF[3][NF], P, float2 out[NF]), acc_cell2(Acc&, const float2 out[NF], P).
#pragma once

#include "f32x2.cuh"
#include "tma_stencil.cuh"

namespace stencil {

// Padded geometry lattice of a face sweep (see above): base, row length Zp,
// rows Yp, planes Xp and entries per field np = Xp Yp Zp.
struct PaddedGeom {
  const void* base;
  int64_t zp, yp, xp, np;
};

template <class P, class = void> struct face_paired { static constexpr bool value = false; };
template <class P> struct face_paired<P, decltype(void(P::PAIRED))> { static constexpr bool value = P::PAIRED; };
template <class P, class = void> struct face_prologue { static constexpr bool value = false; };
template <class P> struct face_prologue<P, decltype(void(&P::prologue))> { static constexpr bool value = true; };

// The physics operations on a thread's VZ cells ([field][cell] arrays), as
// loops over the cells.  Paired physics (PAIR) run a path of their own in the
// kernel, on register pairs.
template <class Phys, int VZ> struct FaceOps {
  static constexpr int NF = Phys::NF, ND = Phys::ND, NG = Phys::NG, NGF = Phys::NGF;
  static constexpr int NDA = ND > 0 ? ND : 1, NGA = NG > 0 ? NG : 1, NGFA = NGF > 0 ? NGF : 1;
  static constexpr bool PAIR = face_paired<Phys>::value && VZ == 2;
  using Params = typename Phys::Params;

  template <int N> __device__ static void col(const float v[][VZ], int j, float* out) {
#pragma unroll
    for (int f = 0; f < N; ++f) out[f] = v[f][j];
  }

  __device__ static void derive(const float q[NF][VZ], float d[NDA][VZ], const Params& P) {
    if constexpr (ND > 0) {
#pragma unroll
      for (int j = 0; j < VZ; ++j) {
        float a[NF], t[NDA];
        col<NF>(q, j, a);
        Phys::derive(a, t, P);
#pragma unroll
        for (int e = 0; e < ND; ++e) d[e][j] = t[e];
      }
    }
  }
  __device__ static void flux(const float L[NF][VZ], const float Ld[NDA][VZ], const float R[NF][VZ],
                              const float Rd[NDA][VZ], const float Sf[NGFA][VZ], int d, const Params& P,
                              float F[NF][VZ]) {
#pragma unroll
    for (int j = 0; j < VZ; ++j) {
      float a[NF], ad[NDA], b[NF], bd[NDA], s[NGFA], o[NF];
      col<NF>(L, j, a);
      col<NDA>(Ld, j, ad);
      col<NF>(R, j, b);
      col<NDA>(Rd, j, bd);
      col<NGFA>(Sf, j, s);
      Phys::flux(a, ad, b, bd, s, d, P, o);
#pragma unroll
      for (int f = 0; f < NF; ++f) F[f][j] = o[f];
    }
  }
  __device__ static void ghost(const float C[NF][VZ], const float Cd[NDA][VZ], const float Sf[NGFA][VZ], int d,
                               float g[NF][VZ], float gd[NDA][VZ]) {
#pragma unroll
    for (int j = 0; j < VZ; ++j) {
      float c[NF], cd[NDA], s[NGFA], gq[NF], gdd[NDA];
      col<NF>(C, j, c);
      col<NDA>(Cd, j, cd);
      col<NGFA>(Sf, j, s);
      Phys::ghost(c, cd, s, d, gq, gdd);
#pragma unroll
      for (int f = 0; f < NF; ++f) g[f][j] = gq[f];
#pragma unroll
      for (int e = 0; e < NDA; ++e) gd[e][j] = gdd[e];
    }
  }
  __device__ static void update(const float C[NF][VZ], const float Cd[NDA][VZ], const float G[NGA][VZ],
                                const float dF[3][NF][VZ], const Params& P, float o[NF][VZ]) {
#pragma unroll
    for (int j = 0; j < VZ; ++j) {
      float c[NF], cd[NDA], gg[NGA], df[3][NF], r[NF];
      col<NF>(C, j, c);
      col<NDA>(Cd, j, cd);
      col<NGA>(G, j, gg);
#pragma unroll
      for (int d = 0; d < 3; ++d) col<NF>(dF[d], j, df[d]);
      Phys::update(c, cd, gg, df, P, r);
#pragma unroll
      for (int f = 0; f < NF; ++f) o[f][j] = r[f];
    }
  }
  __device__ static void acc(typename Phys::Acc& a, const float o[NF][VZ], const Params& P) {
#pragma unroll
    for (int j = 0; j < VZ; ++j) {
      float r[NF];
      col<NF>(o, j, r);
      Phys::acc_cell(a, r, P);
    }
  }
};

template <int TZ, int TY, int S, int NF, int NG, int ND, int VZ> struct FaceLayout {
  static constexpr int RL = TZ + 8;   // state row: 4 halo cells each side (16-byte aligned z origin)
  static constexpr int RR = TY + 2;   // state rows: one halo row each side
  static constexpr int TILE = RL * RR;
  static constexpr int GL = TZ + 4;   // geometry row: 4 halo cells on the low side only
  static constexpr int GR = TY + 1;   // geometry rows: one halo row below
  static constexpr int GTILE = GL * GR;
  static constexpr int G_OFF = (NF * TILE + 31) / 32 * 32;  // 128-byte aligned
  static constexpr int SLOT = (G_OFF + NG * GTILE + 31) / 32 * 32;
  static constexpr uint32_t TX_BYTES = uint32_t(4 * (NF * TILE + NG * GTILE));
  static constexpr uint32_t TX_GEOM = uint32_t(4 * NG * GTILE);
  static constexpr int DSLOT = (ND * TILE + 31) / 32 * 32;  // one buffer of derived values (state tile layout)
  static constexpr size_t SMEM_BYTES = (size_t(S) * SLOT + 2 * size_t(DSLOT)) * 4;
  static constexpr int THREADS = (TZ / VZ) * TY;
};

template <class Phys, int TZ, int TY, int S, int VZ>
__global__ void __launch_bounds__((TZ / VZ) * TY, Phys::MIN_BLOCKS)
    face_sweep_kernel(const __grid_constant__ CUtensorMap tm_q, const __grid_constant__ CUtensorMap tm_g, Geometry g,
                      float* __restrict__ out, typename Phys::Params prm, int* __restrict__ err) {
  constexpr int NF = Phys::NF;
  constexpr int NG = Phys::NG;
  constexpr int NGF = Phys::NGF;
  constexpr int ND = Phys::ND;
  constexpr int NGA = NG > 0 ? NG : 1;
  constexpr int NGFA = NGF > 0 ? NGF : 1;
  constexpr int NDA = ND > 0 ? ND : 1;
  constexpr bool SEL = Phys::SELECT_WALLS;
  using L = FaceLayout<TZ, TY, S, NF, NG, ND, VZ>;
  extern __shared__ __align__(128) float smem[];
  __shared__ __align__(8) uint64_t bars[S];
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
    if constexpr (NG > 0) prefetch_tmap(&tm_g);
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
    uint32_t dyn;
    asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    if (dyn < L::SMEM_BYTES) {
      if (threadIdx.x == 0) atomicExch(err, kErrSmemSize);
      return;
    }
  }
  typename Phys::Params P = prm;

  const int tz = threadIdx.x % (TZ / VZ);
  const int ty = threadIdx.x / (TZ / VZ);
  const int y = y0 + ty;
  const int zb = z0 + VZ * tz;
  const bool active = (y < g.Y) && (zb < g.Z);
  const int kmax = x1 - x0 + 1;  // plane k <-> x = x0 - 1 + k

  // A wait that gives up ends the staging exactly as in the stencil sweep:
  // nothing more is issued, later waits are skipped, the copies in flight are
  // waited for (bounded) before the CTA exits and the error word reports it.
  // Plane -1 (k = 0 of the first chunk) has no state; with geometry its slot
  // receives the ghost plane's geometry only.
  bool bad = false;
  auto issue = [&](int k) {
    const int x = x0 - 1 + k;
    if (bad || k > kmax || x < -1 || x >= g.X || (x < 0 && NG == 0)) return;
    const int s = k % S;
    float* dst = smem + s * L::SLOT;
    mbar_expect_tx(&bars[s], x < 0 ? L::TX_GEOM : L::TX_BYTES);
    last_issued = k;
    if (k == g.missing_plane && blockIdx.x == 0 && blockIdx.y == 0) return;
    if (x >= 0) tma_load_4d(dst, &tm_q, z0 - 4, y0 - 1, x, 0, &bars[s]);
    if constexpr (NG > 0) tma_load_4d(dst + L::G_OFF, &tm_g, z0, y0, x + 1, 0, &bars[s]);
  };
  uint32_t first_issued = 0;  // thread 0: the slots of the first planes actually issued
  if (threadIdx.x == 0)
    for (int k = 0; k < S; ++k) {
      const int before = last_issued;
      issue(k);
      if (last_issued != before) first_issued |= 1u << k;
    }
  // The physics' per-launch set-up (reads of device state such as a clock)
  // runs while the first planes are in flight; a launch with nothing to do
  // lets the copies it issued land before it exits.
  if (!Phys::begin(P)) {
    if (threadIdx.x == 0)
      for (int k = 0; k < S; ++k)
        if ((first_issued >> k) & 1u) mbar_wait_bounded(&bars[k], 0u, g.wait_cycles);
    return;
  }
  // work of the physics that needs no plane, done while the first planes are
  // in flight (every thread of every CTA calls it)
  if constexpr (face_prologue<Phys>::value) Phys::prologue(P);

  uint32_t parity = 0;
  auto wait_plane = [&](int k) {
    const int s = k % S;
    const uint32_t par = (parity >> s) & 1u;
    parity ^= 1u << s;
    if (bad) return;
    if (!mbar_wait_bounded(&bars[s], par, g.wait_cycles)) {
      bad = true;
      if (threadIdx.x == 0) {
        uint32_t d = (parity & 0xffffu) << 16;
        for (int j = k + 1; j <= last_issued; ++j) d |= 1u << (j % S);
        drain = d;
      }
    }
  };
  // offsets of the thread's first cell in a state tile and in a geometry tile
  const int cs = (ty + 1) * L::RL + 4 + VZ * tz;
  const int cg = (ty + 1) * L::GL + 4 + VZ * tz;
  auto state = [&](int k) -> const float* { return smem + (k % S) * L::SLOT; };
  auto geom = [&](int k) -> const float* { return smem + (k % S) * L::SLOT + L::G_OFF; };
  float* const dsm = smem + S * L::SLOT;
  auto dbuf = [&](int k) -> float* { return dsm + (k & 1) * L::DSLOT; };

  using Ops = FaceOps<Phys, VZ>;
  // derived values of plane k for the y/z neighbours: the thread's own cells
  // (from its registers) and one cell of the tile's halo ring per thread
  auto publish = [&](int k, const float d[NDA][VZ]) {
    if constexpr (ND > 0) {
      float* b = dbuf(k);
      if (active) {
#pragma unroll
        for (int e = 0; e < ND; ++e) stv<VZ>(b + e * L::TILE + cs, d[e]);
      }
      const float* base = state(k);
      constexpr int H = 2 * TZ + 2 * TY;
      for (int h = int(threadIdx.x); h < H; h += L::THREADS) {
        int row, z;  // tile row (-1 .. TY) and z offset (-1 .. TZ)
        if (h < TZ) { row = -1; z = h; }
        else if (h < 2 * TZ) { row = TY; z = h - TZ; }
        else if (h < 2 * TZ + TY) { row = h - 2 * TZ; z = -1; }
        else { row = h - 2 * TZ - TY; z = TZ; }
        const int o = (row + 1) * L::RL + 4 + z;
        float q[NF], t[NDA];
#pragma unroll
        for (int f = 0; f < NF; ++f) q[f] = base[f * L::TILE + o];
        Phys::derive(q, t, P);
#pragma unroll
        for (int e = 0; e < ND; ++e) b[e * L::TILE + o] = t[e];
      }
    }
  };
  auto load_state = [&](int k, int off, float v[NF][VZ]) {
    const float* b = state(k);
#pragma unroll
    for (int f = 0; f < NF; ++f) ldv<VZ>(b + f * L::TILE + off, v[f]);
  };
  // The neighbour across a z face, which is a wall for single lanes only:
  // the loaded cell, or the ghost of C (built behind a branch, or always
  // and selected).
  auto across = [&](bool wall, const float C[NF], const float Cd[NDA], const float Sf[NGFA], int d, float nb[NF],
                    float nbd[NDA]) {
    if (SEL || wall) {
      float gq[NF], gd[NDA];
      Phys::ghost(C, Cd, Sf, d, gq, gd);
#pragma unroll
      for (int f = 0; f < NF; ++f) nb[f] = wall ? gq[f] : nb[f];
#pragma unroll
      for (int e = 0; e < NDA; ++e) nbd[e] = wall ? gd[e] : nbd[e];
    }
  };
  // Flux through a face set whose walls are uniform over the warp (x walls
  // over the CTA, y walls over a tile row = one warp): the neighbours R, or
  // the ghosts of C when `wall` (plus = true: C on the minus side).
  auto wall_or = [&](bool wall, bool plus, const float C[NF][VZ], const float Cd[NDA][VZ], const float R[NF][VZ],
                     const float Rd[NDA][VZ], const float Sf[NGFA][VZ], int d, float F[NF][VZ]) {
    if (!wall) {
      if (plus) Ops::flux(C, Cd, R, Rd, Sf, d, P, F);
      else Ops::flux(R, Rd, C, Cd, Sf, d, P, F);
    } else {
      float gq[NF][VZ], gd[NDA][VZ];
      Ops::ghost(C, Cd, Sf, d, gq, gd);
      if (plus) Ops::flux(C, Cd, gq, gd, Sf, d, P, F);
      else Ops::flux(gq, gd, C, Cd, Sf, d, P, F);
    }
  };

  typename Phys::Acc acc;
  Phys::acc_init(acc);
  const long long plane = (long long)g.Y * g.Z;
  const bool ylo = y == 0, yhi = y == g.Y - 1;
  const bool zlo = zb == 0, zhi = zb + VZ - 1 == g.Z - 1;

  if constexpr (Ops::PAIR) {
    // Paired physics, two cells per thread: the state, derived values and
    // fluxes of the thread's cells stay (cell 0, cell 1) register pairs from
    // the 8-byte shared-memory loads to the 8-byte global stores, so the
    // packed instructions need no repacking.
    static_assert(NG == 0 && NGF == 0 && ND > 0, "paired face physics: derived values, no per-cell geometry");
    auto ld2 = [](const float* p) { return *reinterpret_cast<const float2*>(p); };
    auto load2 = [&](const float* b, int off, float2 v[NF]) {
#pragma unroll
      for (int f = 0; f < NF; ++f) v[f] = ld2(b + f * L::TILE + off);
    };
    auto loadd2 = [&](const float* b, int off, float2 v[ND]) {
#pragma unroll
      for (int e = 0; e < ND; ++e) v[e] = ld2(b + e * L::TILE + off);
    };
    auto publish2 = [&](int k, const float2 d[ND]) {
      float dv[NDA][VZ];
#pragma unroll
      for (int e = 0; e < ND; ++e) { dv[e][0] = d[e].x; dv[e][1] = d[e].y; }
      publish(k, dv);
    };
    // one lane (cell j) of a pair as scalars
    auto lane = [](const float2* v, int n, int j, float* o) {
      for (int i = 0; i < n; ++i) o[i] = j ? v[i].y : v[i].x;
    };
    // the ghosts of both cells across a d face
    auto ghost2 = [&](const float2 C[NF], const float2 Cd[ND], int d, float2 gq[NF], float2 gd[ND]) {
      float c[NF], cd[ND], a[NF], ad[ND], b[NF], bd[ND];
      lane(C, NF, 0, c); lane(Cd, ND, 0, cd);
      Phys::ghost(c, cd, nullptr, d, a, ad);
      lane(C, NF, 1, c); lane(Cd, ND, 1, cd);
      Phys::ghost(c, cd, nullptr, d, b, bd);
#pragma unroll
      for (int f = 0; f < NF; ++f) gq[f] = make_float2(a[f], b[f]);
#pragma unroll
      for (int e = 0; e < ND; ++e) gd[e] = make_float2(ad[e], bd[e]);
    };
    float2 Cd2[ND], fx2[NF];
    if (x0 > 0) wait_plane(0);
    wait_plane(1);
    {
      float2 C[NF];
      load2(state(1), cs, C);
      Phys::derive2(C, Cd2, P);
      publish2(1, Cd2);
      if (active) {
        float2 Q[NF], Qd[ND];
        if (x0 > 0) {
          load2(state(0), cs, Q);
          Phys::derive2(Q, Qd, P);
        } else {
          ghost2(C, Cd2, 0, Q, Qd);
        }
        Phys::flux2(Q, Qd, C, Cd2, 0, P, fx2);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      fence_proxy_async();
      issue(S);
    }
    for (int x = x0; x < x1; ++x) {
      const int k = x - x0 + 1;
      const bool xhi = x + 1 >= g.X;
      float2 N[NF], Nd[ND];
      if (!xhi) {
        wait_plane(k + 1);
        load2(state(k + 1), cs, N);
        Phys::derive2(N, Nd, P);
        publish2(k + 1, Nd);
      }
      if (active) {
        const float* cq = state(k);
        const float* db = dbuf(k);
        float2 C[NF], dF[3][NF];
        load2(cq, cs, C);
        {  // x faces: the +x flux of plane k is the -x flux of plane k + 1
          float2 F[NF];
          if (!xhi) {
            Phys::flux2(C, Cd2, N, Nd, 0, P, F);
          } else {
            float2 gq[NF], gd[ND];
            ghost2(C, Cd2, 0, gq, gd);
            Phys::flux2(C, Cd2, gq, gd, 0, P, F);
          }
#pragma unroll
          for (int f = 0; f < NF; ++f) {
            dF[0][f] = f2::sub(F[f], fx2[f]);
            fx2[f] = F[f];
          }
        }
        {  // y faces (walls uniform over the warp)
          float2 Fp[NF], Fm[NF], R[NF], Rd[ND];
          if (!yhi) {
            load2(cq, cs + L::RL, R);
            loadd2(db, cs + L::RL, Rd);
          } else {
            ghost2(C, Cd2, 1, R, Rd);
          }
          Phys::flux2(C, Cd2, R, Rd, 1, P, Fp);
          if (!ylo) {
            load2(cq, cs - L::RL, R);
            loadd2(db, cs - L::RL, Rd);
          } else {
            ghost2(C, Cd2, 1, R, Rd);
          }
          Phys::flux2(R, Rd, C, Cd2, 1, P, Fm);
#pragma unroll
          for (int f = 0; f < NF; ++f) dF[1][f] = f2::sub(Fp[f], Fm[f]);
        }
        {  // z faces: faces 0 and 1 (left cells zl, cell 0) as a pair, face 2 alone
          float a[NF], ad[ND], c[NF], cd[ND];
#pragma unroll
          for (int f = 0; f < NF; ++f) a[f] = cq[f * L::TILE + cs - 1];
#pragma unroll
          for (int e = 0; e < ND; ++e) ad[e] = db[e * L::TILE + cs - 1];
          lane(C, NF, 0, c);
          lane(Cd2, ND, 0, cd);
          across(zlo, c, cd, nullptr, 2, a, ad);
          float2 Lz[NF], Lzd[ND], F01[NF];
#pragma unroll
          for (int f = 0; f < NF; ++f) Lz[f] = make_float2(a[f], C[f].x);
#pragma unroll
          for (int e = 0; e < ND; ++e) Lzd[e] = make_float2(ad[e], Cd2[e].x);
          Phys::flux2(Lz, Lzd, C, Cd2, 2, P, F01);
          float b[NF], bd[ND], F2[NF];
#pragma unroll
          for (int f = 0; f < NF; ++f) b[f] = cq[f * L::TILE + cs + 2];
#pragma unroll
          for (int e = 0; e < ND; ++e) bd[e] = db[e * L::TILE + cs + 2];
          lane(C, NF, 1, c);
          lane(Cd2, ND, 1, cd);
          across(zhi, c, cd, nullptr, 2, b, bd);
          Phys::flux(c, cd, b, bd, nullptr, 2, P, F2);
#pragma unroll
          for (int f = 0; f < NF; ++f) dF[2][f] = f2::sub(make_float2(F01[f].y, F2[f]), F01[f]);
        }
        float2 res[NF];
        Phys::update2(C, Cd2, dF, P, res);
        Phys::acc_cell2(acc, res, P);
        const long long idx = (long long)x * plane + (long long)y * g.Z + zb;
#pragma unroll
        for (int f = 0; f < NF; ++f) *reinterpret_cast<float2*>(out + f * g.n + idx) = res[f];
      }
#pragma unroll
      for (int e = 0; e < ND; ++e) Cd2[e] = Nd[e];
      __syncthreads();
      if (threadIdx.x == 0) {
        fence_proxy_async();
        issue(k + S);
      }
    }
  } else {
  // the first plane's derived values, and the flux through its -x faces
  float Cd[NDA][VZ] = {};
  float fxm[NF][VZ];
  if (x0 > 0 || NG > 0) wait_plane(0);
  wait_plane(1);
  {
    float C[NF][VZ];
    load_state(1, cs, C);
    Ops::derive(C, Cd, P);
    publish(1, Cd);
    if (active) {
      float Sf[NGFA][VZ] = {}, Q[NF][VZ], Qd[NDA][VZ] = {};
      const float* g0 = geom(0);
#pragma unroll
      for (int e = 0; e < NGF; ++e) ldv<VZ>(g0 + e * L::GTILE + cg, Sf[e]);
      if (x0 > 0) {
        load_state(0, cs, Q);
        Ops::derive(Q, Qd, P);
      }
      wall_or(x0 == 0, false, C, Cd, Q, Qd, Sf, 0, fxm);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    fence_proxy_async();
    issue(S);
  }

  for (int x = x0; x < x1; ++x) {
    const int k = x - x0 + 1;
    const bool xhi = x + 1 >= g.X;
    float N[NF][VZ], Nd[NDA][VZ] = {};
    if (!xhi) {
      wait_plane(k + 1);
      load_state(k + 1, cs, N);
      Ops::derive(N, Nd, P);
      publish(k + 1, Nd);
    }
    if (active) {
      float C[NF][VZ], G[NGA][VZ] = {};
      load_state(k, cs, C);
      const float* cgm = geom(k);
#pragma unroll
      for (int e = 0; e < NG; ++e) ldv<VZ>(cgm + e * L::GTILE + cg, G[e]);
      // the geometry of the thread's cells' +d faces
      auto gface = [&](int d, float Sf[NGFA][VZ]) {
#pragma unroll
        for (int e = 0; e < NGFA; ++e)
#pragma unroll
          for (int j = 0; j < VZ; ++j) Sf[e][j] = NGF > 0 ? G[d * NGF + e][j] : 0.f;
      };
      float dF[3][NF][VZ];
      // x faces: the +x flux of plane k is the -x flux of plane k + 1
      {
        float Sx[NGFA][VZ], F[NF][VZ];
        gface(0, Sx);
        wall_or(xhi, true, C, Cd, N, Nd, Sx, 0, F);
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
          for (int j = 0; j < VZ; ++j) {
            dF[0][f][j] = F[f][j] - fxm[f][j];
            fxm[f][j] = F[f][j];
          }
      }
      // y faces: both per cell
      {
        const float* db = dbuf(k);
        float Ym[NF][VZ], Yp[NF][VZ], Ymd[NDA][VZ] = {}, Ypd[NDA][VZ] = {}, Sm[NGFA][VZ] = {}, Sy[NGFA][VZ];
        load_state(k, cs - L::RL, Ym);
        load_state(k, cs + L::RL, Yp);
#pragma unroll
        for (int e = 0; e < ND; ++e) {
          ldv<VZ>(db + e * L::TILE + cs - L::RL, Ymd[e]);
          ldv<VZ>(db + e * L::TILE + cs + L::RL, Ypd[e]);
        }
#pragma unroll
        for (int e = 0; e < NGF; ++e) ldv<VZ>(cgm + (NGF + e) * L::GTILE + cg - L::GL, Sm[e]);
        gface(1, Sy);
        float Fp[NF][VZ], Fm[NF][VZ];
        wall_or(yhi, true, C, Cd, Yp, Ypd, Sy, 1, Fp);
        wall_or(ylo, false, C, Cd, Ym, Ymd, Sm, 1, Fm);
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
          for (int j = 0; j < VZ; ++j) dF[1][f][j] = Fp[f][j] - Fm[f][j];
      }
      // z faces: VZ + 1 for the thread's VZ cells; faces 0 .. VZ-1 (left
      // cells zl, C_0 .. C_{VZ-2}) as one vector call, face VZ alone
      {
        const float* cq = state(k);
        const float* db = dbuf(k);
        float Lz[NF][VZ], Lzd[NDA][VZ] = {}, Sz[NGFA][VZ] = {};
#pragma unroll
        for (int j = 1; j < VZ; ++j) {
#pragma unroll
          for (int f = 0; f < NF; ++f) Lz[f][j] = C[f][j - 1];
#pragma unroll
          for (int e = 0; e < ND; ++e) Lzd[e][j] = Cd[e][j - 1];
#pragma unroll
          for (int e = 0; e < NGF; ++e) Sz[e][j] = G[2 * NGF + e][j - 1];
        }
        {
          float a[NF], ad[NDA] = {}, s[NGFA] = {}, c[NF], cd[NDA];
#pragma unroll
          for (int f = 0; f < NF; ++f) a[f] = cq[f * L::TILE + cs - 1];
#pragma unroll
          for (int e = 0; e < ND; ++e) ad[e] = db[e * L::TILE + cs - 1];
#pragma unroll
          for (int e = 0; e < NGF; ++e) s[e] = cgm[(2 * NGF + e) * L::GTILE + cg - 1];
          Ops::template col<NF>(C, 0, c);
          Ops::template col<NDA>(Cd, 0, cd);
          across(zlo, c, cd, s, 2, a, ad);
#pragma unroll
          for (int f = 0; f < NF; ++f) Lz[f][0] = a[f];
#pragma unroll
          for (int e = 0; e < NDA; ++e) Lzd[e][0] = ad[e];
#pragma unroll
          for (int e = 0; e < NGFA; ++e) Sz[e][0] = s[e];
        }
        float Fz[NF][VZ], Fl[NF];
        Ops::flux(Lz, Lzd, C, Cd, Sz, 2, P, Fz);
        {
          float c[NF], cd[NDA], b[NF], bd[NDA] = {}, s[NGFA] = {};
          Ops::template col<NF>(C, VZ - 1, c);
          Ops::template col<NDA>(Cd, VZ - 1, cd);
#pragma unroll
          for (int f = 0; f < NF; ++f) b[f] = cq[f * L::TILE + cs + VZ];
#pragma unroll
          for (int e = 0; e < ND; ++e) bd[e] = db[e * L::TILE + cs + VZ];
#pragma unroll
          for (int e = 0; e < NGF; ++e) s[e] = G[2 * NGF + e][VZ - 1];
          across(zhi, c, cd, s, 2, b, bd);
          Phys::flux(c, cd, b, bd, s, 2, P, Fl);
        }
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
          for (int j = 0; j < VZ; ++j) dF[2][f][j] = (j + 1 < VZ ? Fz[f][j + 1] : Fl[f]) - Fz[f][j];
      }
      float res[NF][VZ];
      Ops::update(C, Cd, G, dF, P, res);
      Ops::acc(acc, res, P);
      const long long idx = (long long)x * plane + (long long)y * g.Z + zb;
#pragma unroll
      for (int f = 0; f < NF; ++f) stv<VZ>(out + f * g.n + idx, res[f]);
    }
    if constexpr (ND > 0) {
#pragma unroll
      for (int e = 0; e < ND; ++e)
#pragma unroll
        for (int j = 0; j < VZ; ++j) Cd[e][j] = Nd[e][j];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      fence_proxy_async();
      issue(k + S);
    }
  }
  }  // generic path
  if (bad) {
    if (threadIdx.x == 0)
      for (int t = 0; t < S; ++t)
        if ((drain >> t) & 1u) mbar_wait_bounded(&bars[t], (drain >> (16 + t)) & 1u, g.wait_cycles);
    atomicExch(err, kErrWaitTimeout);
  }
  Phys::finish(acc, P, active);
}

}  // namespace stencil
