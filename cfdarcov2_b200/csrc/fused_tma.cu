// Fused single-pass time steps on uniform meshes: heat (d1t(T) = k lapl(T))
// and the first-order acoustic system with Rusanov fluxes.  Each step is ONE
// launch of the TMA sweep (tma_stencil.cuh): state in, state out, one HBM pass.
// Replaces the reference's per-equation JIT kernel (src/fvm3d.cpp:1219-1394),
// which streamed ~180 B/cell of geometry per step; on a uniform mesh the
// geometry reduces to three spacings.
#include <cmath>
#include <cstdlib>
#include <string>

#include "heat_cell.cuh"
#include "tma_host.hpp"

CFDB_MODULE_ANCHOR

namespace {

// Heat: T' = T + dt k sum_d ((T_d+ - T) + (T_d- - T)) / h_d^2.  Boundary faces
// see T_N = T_P (zero gradient, intrinsic to Grad2Var: the reference's _ids
// point to the cell itself, src/mesh3d.cpp:273-276).  FIXED: the cells of
// the box surface then take fixed values (the examples' boundary copy,
// examples/main_3d_heat.cpp:41-60, applied after the step) in the same pass.
struct HeatParams {
  float cx, cy, cz;     // dt k / h_d^2
  const float* fixed;   // surface values (FIXED)
};
template <bool FIXED> struct HeatPhys {
  static constexpr int NF = 1;
  static constexpr int NA = 0;
  static constexpr bool HAS_C = false;
  static constexpr int MIN_BLOCKS = 4;
  using Params = HeatParams;
  struct Acc {};
  __device__ static bool begin(Params&) { return true; }
  __device__ static void ghost(float g[NF], const float p[NF], int) { g[0] = p[0]; }
  __device__ static void cell(const stencil::CellIn<1>& in, const Params& a, float o[NF]) {
    o[0] = heat_update(in.P[0], in.nb[0][0], in.nb[1][0], in.nb[2][0], in.nb[3][0], in.nb[4][0], in.nb[5][0], a.cx,
                       a.cy, a.cz);
    // (loading the wall values one plane ahead instead, only where walls
    // are, measured 3.88 against 3.83 ms per 200 steps at 200^3)
    if (FIXED && in.walls) o[0] = a.fixed[in.idx];
  }
  __device__ static void acc_init(Acc&) {}
  __device__ static void acc_cell(Acc&, const float*, const Params&) {}
  __device__ static void finish(Acc&, const Params&, bool) {}
};

// Leapfrog of d2t(u) = k sum_j L_{m_j}(u) on an exact lattice, the equation
// the reference's wave example builds (examples/main_3d_wave.cu:
// d2t(u) = c^2 (d2dx(u) + d2dy(u))), with the operands in the order of the
// operator kernels and the generated ones (Grad2Var, src/fvm3d.cpp:831-906;
// update, src/fvm3d.cpp:710-765), every operation rounded on its own:
//   sn_f  = (u_N(f) - u) alpha_f                      face slots f = 0..5
//   acc_d = 0 + sum_{f: n_{f,d} != 0} (sn_f n_{f,d}) A_f,   L_m = 0 + sum_{d in m} acc_d / V
//   R = k ((L_m1 + L_m2) + L_m3)
//   first step: u' = dt R + u;  later: u' = (dt dt R + 2 u) - u_prev
// A boundary face has u_N = u: its sn is +0 whatever alpha the wall has, so
// the interior alphas serve every face.  u_prev comes one plane ahead from
// global memory (HAS_PRE); only u is staged with its halo.  Each direction's
// nonzero normals are its own two faces (the uniform meshes the sweep serves
// are axis-aligned).  GEOM says how the face factors round: D2T_DIVIDE
// divides by V; D2T_RECIP multiplies by 1/V where that is exact (V a power of
// two: acc / V == acc * (1/V) bit for bit); D2T_UNIT has alpha, the normals on
// their own faces, the areas and V all exactly 1 (unit cells), where every
// product by them returns its operand, so they are left out.  FORM >= 0 packs the term masks at compile time (3 bits
// each: 7 = lapl, 1 | 2 << 3 = d2dx + d2dy, ...), so the sum has no branches;
// FORM < 0 reads them from the parameters.  Directions no term uses are
// skipped.
struct D2tParams {
  float* prev;      // u at the previous step (the first step reads u again: no subtraction)
  float alpha[6];   // interior alpha per face slot
  float nrm[3][6];  // normal component d of face slot f
  float area[6];
  float volume, vinv, k, dt;
  int masks[3];     // direction mask of each term
  int n_terms;
  int used;         // union of the masks
  int first;
};
enum { D2T_DIVIDE = 0, D2T_RECIP = 1, D2T_UNIT = 2 };
template <int GEOM, int FORM> struct D2tPhys {
  static constexpr int NF = 1;
  static constexpr int NA = 0;
  static constexpr bool HAS_C = false;
  static constexpr bool HAS_PRE = true;
  static constexpr int MIN_BLOCKS = 4;
  using Params = D2tParams;
  struct Acc {};
  static constexpr int form_mask(int j) { return (FORM >> (3 * j)) & 7; }
  __device__ static int term_mask(const Params& a, int j) { return FORM >= 0 ? form_mask(j) : a.masks[j]; }
  __device__ static int terms(const Params& a) {
    return FORM >= 0 ? (form_mask(0) != 0) + (form_mask(1) != 0) + (form_mask(2) != 0) : a.n_terms;
  }
  __device__ static int used(const Params& a) {
    return FORM >= 0 ? (form_mask(0) | form_mask(1) | form_mask(2)) : a.used;
  }
  __device__ static float* pre_ptr(const Params& a) { return a.prev; }
  __device__ static bool begin(Params&) { return true; }
  __device__ static void ghost(float g[NF], const float p[NF], int) { g[0] = p[0]; }
  __device__ static void cell(const stencil::CellIn<1>& in, const Params& a, float o[NF]) {
    const float u = in.P[0];
    // sweep neighbour order x-, x+, y-, y+, z-, z+ by face slot (0/1 z, 2/3 y, 4/5 x)
    constexpr int nb_of_slot[6] = {4, 5, 2, 3, 0, 1};
    float L[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (!((used(a) >> d) & 1)) continue;
      float acc = 0.f;
      const int f0 = 4 - 2 * d;  // the direction's - and + faces, in slot order
#pragma unroll
      for (int f = f0; f < f0 + 2; ++f) {
        const float diff = __fsub_rn(in.nb[nb_of_slot[f]][0], u);
        if (GEOM == D2T_UNIT) acc = __fadd_rn(acc, diff);
        else acc = __fadd_rn(acc, __fmul_rn(__fmul_rn(__fmul_rn(diff, a.alpha[f]), a.nrm[d][f]), a.area[f]));
      }
      L[d] = GEOM == D2T_UNIT ? acc : GEOM == D2T_RECIP ? __fmul_rn(acc, a.vinv) : __fdiv_rn(acc, a.volume);
    }
    float S = 0.f;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      if (j >= terms(a)) break;
      float t = 0.f;
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if ((term_mask(a, j) >> d) & 1) t = __fadd_rn(t, L[d]);
      S = j == 0 ? t : __fadd_rn(S, t);
    }
    const float R = __fmul_rn(a.k, S);
    o[0] = a.first ? __fadd_rn(__fmul_rn(a.dt, R), u)
                   : __fsub_rn(__fadd_rn(__fmul_rn(__fmul_rn(a.dt, a.dt), R), __fmul_rn(2.0f, u)), in.pre);
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

// Tile width of the wave-template sweeps and of the heat sweep with the
// boundary copy: 64 where it pads the z rows less than 128 (nz = 400: 448
// against 512 cells per row; 126 against 156 us per d2t step, 158 against
// 176 us per heat step with the copy), else as dispatch_tz.  The plain heat
// sweep keeps 128 at nz = 400 (112 us against 123 us with 64).
template <class Phys>
int dispatch_padded(cfdb_ctx* ctx, const cfdb_mesh* m, const void* u, void* u_next, const typename Phys::Params& prm) {
  const int64_t pad64 = (m->nz + 63) / 64 * 64, pad128 = (m->nz + 127) / 128 * 128;
  if (m->nz >= 128 && pad64 < pad128)
    return stencil::launch_sweep<Phys, 64, 8, 6>(ctx, m, u, nullptr, nullptr, u_next, prm, 0);
  return dispatch_tz<Phys, 6>(ctx, m, u, u_next, nullptr, prm, 0);
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

int fused_heat_step(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* T, void* Tn, double k, double dt,
                    const void* fixed) {
  if (dtype != CFDB_F32) return cfdb_fail(ctx, CFDB_EUNSUPPORTED, "the fused heat step computes in float32 only");
  if (int rc = stencil::check_sweep(ctx, m, {T, Tn})) return rc;
  HeatParams p;
  p.cx = float(dt * k / (m->dx * m->dx));
  p.cy = float(dt * k / (m->dy * m->dy));
  p.cz = float(dt * k / (m->dz * m->dz));
  p.fixed = static_cast<const float*>(fixed);
  if (fixed) return dispatch_padded<HeatPhys<true>>(ctx, m, T, Tn, p);
  // 128x24 tiles with 4 slots once rows are 128 wide: 768 threads (24 rows
  // of 32, four z cells each), two CTAs per SM, 8 % y halo: 0.90 of HBM at
  // 512^3 and 0.94 at 384^3 against 0.71 and 0.75 with 128x8 tiles and 6
  // slots, the same at 256^3 (128x32: 0.74, 128x16: 0.70, 128x12: 0.78 at
  // 512^3).  The heat step with the boundary copy keeps its tiles (taller
  // ones measured slower there: 24 against 21 us per 200^3 step).
  if (m->nz >= 128)
    return stencil::launch_sweep<HeatPhys<false>, 128, 24, 4>(ctx, m, T, nullptr, nullptr, Tn, p, 0);
  return dispatch_tz<HeatPhys<false>, 6>(ctx, m, T, Tn, nullptr, p, 0);
}

int fused_d2t_step(cfdb_ctx* ctx, cfdb_mesh* m, const void* u, const void* u_prev, void* u_next, double k,
                   const int32_t* masks, int32_t n_terms, double dt, int first_step) {
  if (int rc = stencil::check_sweep(ctx, m, {u, u_prev, u_next})) return rc;
  cfdb_lattice_geometry lat{};
  if (int rc = cfdb_mesh_lattice_geometry(m, &lat)) return rc;
  if (!lat.exact)
    return cfdb_fail(ctx, CFDB_EUNSUPPORTED,
                     "cfdb_d2t_step: the mesh is not an exact lattice (its FP32 face values differ between cells)");
  D2tParams p{};
  p.prev = const_cast<float*>(static_cast<const float*>(first_step ? u : u_prev));
  for (int f = 0; f < 6; ++f) {
    p.alpha[f] = lat.alpha[f];
    p.area[f] = lat.area[f];
  }
  for (int d = 0; d < 3; ++d) {
    int faces = 0;  // bit f: n_{f,d} != 0
    for (int f = 0; f < 6; ++f) {
      p.nrm[d][f] = lat.normal[d * 6 + f];
      if (lat.normal[d * 6 + f] != 0.f) faces |= 1 << f;
    }
    if (faces != (3 << (4 - 2 * d)))
      return cfdb_fail(ctx, CFDB_EUNSUPPORTED, "cfdb_d2t_step: direction %d has normals off its own two faces", d);
  }
  p.volume = lat.volume;
  int e2 = 0;
  const bool recip = lat.volume > 0.f && std::frexp(double(lat.volume), &e2) == 0.5 && std::isnormal(1.0f / lat.volume);
  p.vinv = recip ? 1.0f / lat.volume : 0.f;
  p.k = float(k);
  p.dt = float(dt);
  p.n_terms = n_terms;
  for (int j = 0; j < 3; ++j) {
    p.masks[j] = j < n_terms ? masks[j] : 0;
    p.used |= p.masks[j];
  }
  p.first = first_step ? 1 : 0;
  bool unit = lat.volume == 1.f;
  for (int f = 0; f < 6; ++f) unit = unit && lat.alpha[f] == 1.f && lat.area[f] == 1.f && lat.normal[(f < 2 ? 2 : f < 4 ? 1 : 0) * 6 + f] == 1.f;
  const int form = p.masks[0] | p.masks[1] << 3 | p.masks[2] << 6;
  // the reference's wave equation (d2dx + d2dy), lapl, and d2dx + d2dy + d2dz
  // compiled with their masks
  constexpr int XY = 1 | 2 << 3, LAPL = 7, XYZ = 1 | 2 << 3 | 4 << 6;
  if (unit) {
    if (form == XY) return dispatch_padded<D2tPhys<D2T_UNIT, XY>>(ctx, m, u, u_next, p);
    if (form == LAPL) return dispatch_padded<D2tPhys<D2T_UNIT, LAPL>>(ctx, m, u, u_next, p);
    if (form == XYZ) return dispatch_padded<D2tPhys<D2T_UNIT, XYZ>>(ctx, m, u, u_next, p);
    return dispatch_padded<D2tPhys<D2T_UNIT, -1>>(ctx, m, u, u_next, p);
  }
  if (recip) {
    if (form == XY) return dispatch_padded<D2tPhys<D2T_RECIP, XY>>(ctx, m, u, u_next, p);
    if (form == LAPL) return dispatch_padded<D2tPhys<D2T_RECIP, LAPL>>(ctx, m, u, u_next, p);
    return dispatch_padded<D2tPhys<D2T_RECIP, -1>>(ctx, m, u, u_next, p);
  }
  return dispatch_padded<D2tPhys<D2T_DIVIDE, -1>>(ctx, m, u, u_next, p);
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
