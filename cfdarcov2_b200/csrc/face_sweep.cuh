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
// (array extents of size 0 are passed as 1).
#pragma once

#include "tma_stencil.cuh"

namespace stencil {

// Padded geometry lattice of a face sweep (see above): base, row length Zp,
// rows Yp, planes Xp and entries per field np = Xp Yp Zp.
struct PaddedGeom {
  const void* base;
  int64_t zp, yp, xp, np;
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
  if (!Phys::begin(P)) return;

  const int tz = threadIdx.x % (TZ / VZ);
  const int ty = threadIdx.x / (TZ / VZ);
  const int y = y0 + ty;
  const int zb = z0 + VZ * tz;
  const bool active = (y < g.Y) && (zb < g.Z);
  const int kmax = x1 - x0 + 1;  // plane k <-> x = x0 - 1 + k

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
    last_issued = -1;
    drain = 0;
  }
  __syncthreads();

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
  if (threadIdx.x == 0)
    for (int k = 0; k < S; ++k) issue(k);

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

  auto derive_v = [&](const float v[NF][VZ], float d[NDA][VZ]) {
    if constexpr (ND > 0) {
#pragma unroll
      for (int j = 0; j < VZ; ++j) {
        float q[NF], t[NDA];
#pragma unroll
        for (int f = 0; f < NF; ++f) q[f] = v[f][j];
        Phys::derive(q, t, P);
#pragma unroll
        for (int e = 0; e < ND; ++e) d[e][j] = t[e];
      }
    }
  };
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
  // The ghosts of a thread's VZ cells across their d faces with geometry Sf;
  // used behind a branch that is uniform over the CTA (x walls) or the warp
  // (y walls, a tile row being one warp), so no lane diverges.
  auto ghost_v = [&](const float C[NF][VZ], const float Cd[NDA][VZ], const float Sf[NGFA][VZ], int d,
                     float nb[NF][VZ], float nbd[NDA][VZ]) {
#pragma unroll
    for (int j = 0; j < VZ; ++j) {
      float c[NF], cd[NDA], s[NGFA], gq[NF], gd[NDA];
#pragma unroll
      for (int f = 0; f < NF; ++f) c[f] = C[f][j];
#pragma unroll
      for (int e = 0; e < NDA; ++e) cd[e] = ND > 0 ? Cd[e][j] : 0.f;
#pragma unroll
      for (int e = 0; e < NGFA; ++e) s[e] = NGF > 0 ? Sf[e][j] : 0.f;
      Phys::ghost(c, cd, s, d, gq, gd);
#pragma unroll
      for (int f = 0; f < NF; ++f) nb[f][j] = gq[f];
#pragma unroll
      for (int e = 0; e < NDA; ++e) nbd[e][j] = gd[e];
    }
  };
  // The neighbour across a z face, which is a wall for single lanes only: the
  // loaded cell, or the ghost of C (built behind a branch, or always and
  // selected).
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

  // the first plane's derived values, and the flux through its -x faces
  float Cd[NDA][VZ] = {};
  float fxm[NF][VZ];
  if (x0 > 0 || NG > 0) wait_plane(0);
  wait_plane(1);
  {
    float C[NF][VZ];
    load_state(1, cs, C);
    derive_v(C, Cd);
    publish(1, Cd);
    if (active) {
      float Sf[NGFA][VZ] = {}, Q[NF][VZ], Qd[NDA][VZ] = {};
      const float* g0 = geom(0);
#pragma unroll
      for (int e = 0; e < NGF; ++e) ldv<VZ>(g0 + e * L::GTILE + cg, Sf[e]);
      if (x0 > 0) {
        load_state(0, cs, Q);
        derive_v(Q, Qd);
      } else {
        ghost_v(C, Cd, Sf, 0, Q, Qd);
      }
#pragma unroll
      for (int j = 0; j < VZ; ++j) {
        float a[NF], ad[NDA], b[NF], bd[NDA], s[NGFA], F[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) { b[f] = C[f][j]; a[f] = Q[f][j]; }
#pragma unroll
        for (int e = 0; e < NDA; ++e) { bd[e] = Cd[e][j]; ad[e] = Qd[e][j]; }
#pragma unroll
        for (int e = 0; e < NGFA; ++e) s[e] = NGF > 0 ? Sf[e][j] : 0.f;
        Phys::flux(a, ad, b, bd, s, 0, P, F);
#pragma unroll
        for (int f = 0; f < NF; ++f) fxm[f][j] = F[f];
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    fence_proxy_async();
    issue(S);
  }

  typename Phys::Acc acc;
  Phys::acc_init(acc);
  const long long plane = (long long)g.Y * g.Z;
  const bool ylo = y == 0, yhi = y == g.Y - 1;
  const bool zlo = zb == 0, zhi = zb + VZ - 1 == g.Z - 1;

  for (int x = x0; x < x1; ++x) {
    const int k = x - x0 + 1;
    const bool xhi = x + 1 >= g.X;
    float N[NF][VZ], Nd[NDA][VZ] = {};
    if (!xhi) {
      wait_plane(k + 1);
      load_state(k + 1, cs, N);
      derive_v(N, Nd);
      publish(k + 1, Nd);
    }
    if (active) {
      float C[NF][VZ], G[NGA][VZ];
      load_state(k, cs, C);
      const float* cgm = geom(k);
#pragma unroll
      for (int e = 0; e < NG; ++e) ldv<VZ>(cgm + e * L::GTILE + cg, G[e]);
      auto cell = [&](int j, float c[NF], float cd[NDA], float gg[NGA]) {
#pragma unroll
        for (int f = 0; f < NF; ++f) c[f] = C[f][j];
#pragma unroll
        for (int e = 0; e < NDA; ++e) cd[e] = Cd[e][j];
#pragma unroll
        for (int e = 0; e < NGA; ++e) gg[e] = G[e][j];
      };
      // the geometry of the thread's cells' +d faces
      auto gface = [&](int d, float Sf[NGFA][VZ]) {
#pragma unroll
        for (int e = 0; e < NGFA; ++e)
#pragma unroll
          for (int j = 0; j < VZ; ++j) Sf[e][j] = NGF > 0 ? G[d * NGF + e][j] : 0.f;
      };
      float dF[VZ][3][NF];
      // x faces
      float Sx[NGFA][VZ];
      gface(0, Sx);
      if (xhi) ghost_v(C, Cd, Sx, 0, N, Nd);
#pragma unroll
      for (int j = 0; j < VZ; ++j) {
        float c[NF], cd[NDA], gg[NGA], b[NF], bd[NDA], s[NGFA], F[NF];
        cell(j, c, cd, gg);
#pragma unroll
        for (int f = 0; f < NF; ++f) b[f] = N[f][j];
#pragma unroll
        for (int e = 0; e < NDA; ++e) bd[e] = Nd[e][j];
#pragma unroll
        for (int e = 0; e < NGFA; ++e) s[e] = Sx[e][j];
        Phys::flux(c, cd, b, bd, s, 0, P, F);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          dF[j][0][f] = F[f] - fxm[f][j];
          fxm[f][j] = F[f];
        }
      }
      // y faces
      {
        const float* db = dbuf(k);
        float Ym[NF][VZ], Yp[NF][VZ], Ymd[NDA][VZ] = {}, Ypd[NDA][VZ] = {}, Sm[NGFA][VZ] = {};
        load_state(k, cs - L::RL, Ym);
        load_state(k, cs + L::RL, Yp);
#pragma unroll
        for (int e = 0; e < ND; ++e) {
          ldv<VZ>(db + e * L::TILE + cs - L::RL, Ymd[e]);
          ldv<VZ>(db + e * L::TILE + cs + L::RL, Ypd[e]);
        }
#pragma unroll
        for (int e = 0; e < NGF; ++e) ldv<VZ>(cgm + (NGF + e) * L::GTILE + cg - L::GL, Sm[e]);
        float Sy[NGFA][VZ];
        gface(1, Sy);
        if (yhi) ghost_v(C, Cd, Sy, 1, Yp, Ypd);
        if (ylo) ghost_v(C, Cd, Sm, 1, Ym, Ymd);
#pragma unroll
        for (int j = 0; j < VZ; ++j) {
          float c[NF], cd[NDA], gg[NGA], Fp[NF], Fm[NF];
          cell(j, c, cd, gg);
          {
            float b[NF], bd[NDA], s[NGFA];
#pragma unroll
            for (int f = 0; f < NF; ++f) b[f] = Yp[f][j];
#pragma unroll
            for (int e = 0; e < NDA; ++e) bd[e] = Ypd[e][j];
#pragma unroll
            for (int e = 0; e < NGFA; ++e) s[e] = Sy[e][j];
            Phys::flux(c, cd, b, bd, s, 1, P, Fp);
          }
          {
            float a[NF], ad[NDA], s[NGFA];
#pragma unroll
            for (int f = 0; f < NF; ++f) a[f] = Ym[f][j];
#pragma unroll
            for (int e = 0; e < NDA; ++e) ad[e] = Ymd[e][j];
#pragma unroll
            for (int e = 0; e < NGFA; ++e) s[e] = Sm[e][j];
            Phys::flux(a, ad, c, cd, s, 1, P, Fm);
          }
#pragma unroll
          for (int f = 0; f < NF; ++f) dF[j][1][f] = Fp[f] - Fm[f];
        }
      }
      // z faces: VZ + 1 for the thread's VZ cells
      {
        const float* cq = state(k);
        const float* db = dbuf(k);
        float Fz[VZ + 1][NF];
        {
          float c[NF], cd[NDA], gg[NGA], a[NF], ad[NDA], s[NGFA];
          cell(0, c, cd, gg);
#pragma unroll
          for (int f = 0; f < NF; ++f) a[f] = cq[f * L::TILE + cs - 1];
#pragma unroll
          for (int e = 0; e < NDA; ++e) ad[e] = ND > 0 ? db[e * L::TILE + cs - 1] : 0.f;
#pragma unroll
          for (int e = 0; e < NGFA; ++e) s[e] = NGF > 0 ? cgm[(2 * NGF + e) * L::GTILE + cg - 1] : 0.f;
          across(zlo, c, cd, s, 2, a, ad);
          Phys::flux(a, ad, c, cd, s, 2, P, Fz[0]);
        }
#pragma unroll
        for (int j = 1; j < VZ; ++j) {
          float a[NF], ad[NDA], ga[NGA], b[NF], bd[NDA], gb[NGA], s[NGFA];
          cell(j - 1, a, ad, ga);
          cell(j, b, bd, gb);
#pragma unroll
          for (int e = 0; e < NGFA; ++e) s[e] = NGF > 0 ? ga[2 * NGF + e] : 0.f;
          Phys::flux(a, ad, b, bd, s, 2, P, Fz[j]);
        }
        {
          float c[NF], cd[NDA], gg[NGA], b[NF], bd[NDA], s[NGFA];
          cell(VZ - 1, c, cd, gg);
#pragma unroll
          for (int f = 0; f < NF; ++f) b[f] = cq[f * L::TILE + cs + VZ];
#pragma unroll
          for (int e = 0; e < NDA; ++e) bd[e] = ND > 0 ? db[e * L::TILE + cs + VZ] : 0.f;
#pragma unroll
          for (int e = 0; e < NGFA; ++e) s[e] = NGF > 0 ? gg[2 * NGF + e] : 0.f;
          across(zhi, c, cd, s, 2, b, bd);
          Phys::flux(c, cd, b, bd, s, 2, P, Fz[VZ]);
        }
#pragma unroll
        for (int j = 0; j < VZ; ++j)
#pragma unroll
          for (int f = 0; f < NF; ++f) dF[j][2][f] = Fz[j + 1][f] - Fz[j][f];
      }
      float res[NF][VZ];
#pragma unroll
      for (int j = 0; j < VZ; ++j) {
        float c[NF], cd[NDA], gg[NGA], o[NF];
        cell(j, c, cd, gg);
        Phys::update(c, cd, gg, dF[j], P, o);
        Phys::acc_cell(acc, o, P);
#pragma unroll
        for (int f = 0; f < NF; ++f) res[f][j] = o[f];
      }
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
  if (bad) {
    if (threadIdx.x == 0)
      for (int t = 0; t < S; ++t)
        if ((drain >> t) & 1u) mbar_wait_bounded(&bars[t], (drain >> (16 + t)) & 1u, g.wait_cycles);
    atomicExch(err, kErrWaitTimeout);
  }
  Phys::finish(acc, P, active);
}

}  // namespace stencil
