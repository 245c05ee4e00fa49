// Fused single-pass time steps on uniform meshes: heat (d1t(T) = k lapl(T))
// and the first-order acoustic system with Rusanov fluxes.  Each step is ONE
// launch of the TMA sweep (tma_stencil.cuh): state in, state out, one HBM pass.
// Replaces the reference's per-equation JIT kernel (src/fvm3d.cpp:1219-1394),
// which streamed ~180 B/cell of geometry per step; on a uniform mesh the
// geometry reduces to three spacings.
#include <cstdlib>
#include <string>

#include "heat_cell.cuh"
#include "tma_host.hpp"

CFDB_MODULE_ANCHOR

namespace {

// Heat: T' = T + dt k sum_d ((T_d+ - T) + (T_d- - T)) / h_d^2.  Boundary faces
// see T_N = T_P (zero gradient, intrinsic to Grad2Var: the reference's _ids
// point to the cell itself, src/mesh3d.cpp:273-276).
struct HeatPhys {
  static constexpr int NF = 1;
  static constexpr int NA = 0;
  static constexpr bool HAS_C = false;
  static constexpr int MIN_BLOCKS = 4;
  struct Params { float cx, cy, cz; };  // dt k / h_d^2
  struct Acc {};
  __device__ static bool begin(Params&) { return true; }
  __device__ static void ghost(float g[NF], const float p[NF], int) { g[0] = p[0]; }
  __device__ static void cell(const stencil::CellIn<1>& in, const Params& a, float o[NF]) {
    o[0] = heat_update(in.P[0], in.nb[0][0], in.nb[1][0], in.nb[2][0], in.nb[3][0], in.nb[4][0], in.nb[5][0], a.cx,
                       a.cy, a.cz);
  }
  __device__ static void acc_init(Acc&) {}
  __device__ static void acc_cell(Acc&, const float*, const Params&) {}
  __device__ static void finish(Acc&, const Params&, bool) {}
};

// Acoustic system (p, u, v, w), rho = 1, Rusanov face flux on a uniform mesh:
//   R_p   = -sum_d ih_d [c_P^2 (u_d+ - u_d-)/2 - hc+ (p+ - p) - hc- (p- - p)]
//   R_u_e = -sum_d ih_d [delta_ed (p+ - p-)/2 - hc+ (u_e+ - u_e) - hc- (u_e- - u_e)]
// with hc = c_f / 2 and c_f = max(c_P, c_N) (mode 0) or (c_P + c_N)/2
// (mode 1).  Reflective walls: ghost = P with the wall-normal velocity negated.
template <bool C_FIELD> struct WavePhys {
  static constexpr int NF = 4;
  static constexpr int NA = 0;
  static constexpr bool HAS_C = C_FIELD;
  static constexpr int FT = C_FIELD ? 5 : 4;
  static constexpr int MIN_BLOCKS = 2;
  // k2[d] = dt c^2 ih_d / 2, kc[d] = dt c ih_d / 2, kp[d] = dt ih_d / 2 (constant c)
  struct Params { float dt, ih[3], c; int mode; float k2[3], kc[3], kp[3]; };
  struct Acc {};
  __device__ static bool begin(Params&) { return true; }
  __device__ static void ghost(float g[FT], const float p[FT], int dir) {
#pragma unroll
    for (int f = 0; f < FT; ++f) g[f] = p[f];
    g[1 + dir] = -p[1 + dir];
  }
  __device__ static void cell(const stencil::CellIn<FT>& in, const Params& a, float o[NF]) {
    const float* P = in.P;
    if (!C_FIELD) {
      // constant c: the Rusanov dissipation is a 7-point Laplacian with weight c/2
      //   p'   = p   - sum_d [k2_d (u_d+ - u_d-) - kc_d (p_d+ + p_d- - 2p)]
      //   u_e' = u_e - kp_e (p_e+ - p_e-) + sum_d kc_d (u_e,d+ + u_e,d- - 2 u_e)
      float op = P[0], ou[3] = {P[1], P[2], P[3]};
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float* m = in.nb[2 * d];
        const float* p = in.nb[2 * d + 1];
        op -= a.k2[d] * (p[1 + d] - m[1 + d]) - a.kc[d] * ((p[0] + m[0]) - 2.0f * P[0]);
        ou[d] -= a.kp[d] * (p[0] - m[0]);
#pragma unroll
        for (int e = 0; e < 3; ++e) ou[e] += a.kc[d] * ((p[1 + e] + m[1 + e]) - 2.0f * P[1 + e]);
      }
      o[0] = op; o[1] = ou[0]; o[2] = ou[1]; o[3] = ou[2];
      return;
    }
    const float cP = C_FIELD ? P[FT - 1] : a.c;
    const float c2 = cP * cP;
    float rp = 0.f, ru[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float* m = in.nb[2 * d];
      const float* p = in.nb[2 * d + 1];
      float hm, hp;
      if (C_FIELD) {
        const float cm = m[FT - 1], cpl = p[FT - 1];
        hm = 0.5f * (a.mode == 0 ? fmaxf(cP, cm) : 0.5f * (cP + cm));
        hp = 0.5f * (a.mode == 0 ? fmaxf(cP, cpl) : 0.5f * (cP + cpl));
      } else {
        hm = hp = 0.5f * a.c;
      }
      const float ih = a.ih[d];
      rp -= ih * (c2 * 0.5f * (p[1 + d] - m[1 + d]) - hp * (p[0] - P[0]) - hm * (m[0] - P[0]));
#pragma unroll
      for (int e = 0; e < 3; ++e) {
        float t = -hp * (p[1 + e] - P[1 + e]) - hm * (m[1 + e] - P[1 + e]);
        if (e == d) t += 0.5f * (p[0] - m[0]);
        ru[e] -= ih * t;
      }
    }
    o[0] = P[0] + a.dt * rp;
    o[1] = P[1] + a.dt * ru[0];
    o[2] = P[2] + a.dt * ru[1];
    o[3] = P[3] + a.dt * ru[2];
  }
  __device__ static void acc_init(Acc&) {}
  __device__ static void acc_cell(Acc&, const float*, const Params&) {}
  __device__ static void finish(Acc&, const Params&, bool) {}
};

template <class Phys, int S>
int dispatch_tz(cfdb_ctx* ctx, const cfdb_mesh* m, const void* q, void* out, const void* c,
                const typename Phys::Params& prm, int ctas_per_sm) {
  if (m->nz >= 128) return stencil::launch_sweep<Phys, 128, 8, S>(ctx, m, q, nullptr, c, out, prm, ctas_per_sm);
  if (m->nz >= 64) return stencil::launch_sweep<Phys, 64, 8, S>(ctx, m, q, nullptr, c, out, prm, ctas_per_sm);
  return stencil::launch_sweep<Phys, 32, 8, S>(ctx, m, q, nullptr, c, out, prm, ctas_per_sm);
}

// Tile shape of the constant-c wave sweep.  CFDB_WAVE_TILE=TZxTYxS picks one of
// the instantiated shapes (for tuning sweeps); the default is 128x8x3 (three
// staged planes: the shape that measured fastest on meshes beyond L2).
int dispatch_wave_tiles(cfdb_ctx* ctx, const cfdb_mesh* m, const void* q, void* qn,
                        const WavePhys<false>::Params& p) {
  using W = WavePhys<false>;
  static const char* env = getenv("CFDB_WAVE_TILE");
  const std::string t = env ? env : "";
  if (m->nz >= 128) {
    if (t == "128x4x4") return stencil::launch_sweep<W, 128, 4, 4>(ctx, m, q, nullptr, nullptr, qn, p, 0);
    if (t == "128x8x4") return stencil::launch_sweep<W, 128, 8, 4>(ctx, m, q, nullptr, nullptr, qn, p, 0);
    if (t == "64x8x4") return stencil::launch_sweep<W, 64, 8, 4>(ctx, m, q, nullptr, nullptr, qn, p, 0);
    if (t == "128x8x4v2") return stencil::launch_sweep<W, 128, 8, 4, 2>(ctx, m, q, nullptr, nullptr, qn, p, 0);
    if (t == "64x8x4v1") return stencil::launch_sweep<W, 64, 8, 4, 1>(ctx, m, q, nullptr, nullptr, qn, p, 0);
  }
  if (m->nz >= 128) return stencil::launch_sweep<W, 128, 8, 3>(ctx, m, q, nullptr, nullptr, qn, p, 0);
  return dispatch_tz<W, 4>(ctx, m, q, qn, nullptr, p, 0);
}

}  // namespace

int fused_heat_step(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* T, void* Tn, double k, double dt) {
  if (dtype != CFDB_F32) return cfdb_fail(ctx, CFDB_EUNSUPPORTED, "the fused heat step computes in float32 only");
  if (int rc = stencil::check_sweep(ctx, m, {T, Tn})) return rc;
  HeatPhys::Params p;
  p.cx = float(dt * k / (m->dx * m->dx));
  p.cy = float(dt * k / (m->dy * m->dy));
  p.cz = float(dt * k / (m->dz * m->dz));
  return dispatch_tz<HeatPhys, 6>(ctx, m, T, Tn, nullptr, p, 0);
}

int fused_wave_step(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* q, void* qn, const void* c, double cconst,
                    int mode, double dt) {
  if (dtype != CFDB_F32) return cfdb_fail(ctx, CFDB_EUNSUPPORTED, "the fused wave step computes in float32 only");
  if (int rc = stencil::check_sweep(ctx, m, {q, qn, c})) return rc;
  const double ih[3] = {1.0 / m->dx, 1.0 / m->dy, 1.0 / m->dz};
  if (c) {
    WavePhys<true>::Params p{float(dt), {float(ih[0]), float(ih[1]), float(ih[2])}, 0.f, mode, {}, {}, {}};
    return dispatch_tz<WavePhys<true>, 4>(ctx, m, q, qn, c, p, 0);
  }
  WavePhys<false>::Params p{float(dt), {float(ih[0]), float(ih[1]), float(ih[2])}, float(cconst), mode, {}, {}, {}};
  for (int d = 0; d < 3; ++d) {
    p.k2[d] = float(0.5 * dt * cconst * cconst * ih[d]);
    p.kc[d] = float(0.5 * dt * cconst * ih[d]);
    p.kp[d] = float(0.5 * dt * ih[d]);
  }
  return dispatch_wave_tiles(ctx, m, q, qn, p);
}
