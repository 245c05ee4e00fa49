// fv_oracle.hpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// CPU restatement of cfdARCO's finite-volume time step, templated on the
// working precision (float = the reference's own precision, double = the
// FP64 oracle every GPU result is compared against).  Only tests/, the smoke
// check and bench.py's CPU-baseline leg may load this code.
//
// Parity status: UNPINNED.  The reference (int0vrt/cfdARCOV2) cannot be built
// here (Eigen3, OCCA, RMM, MPI, VTK are absent and there is no network) and it
// ships no tests or golden vectors.  This restatement is pinned instead by
// analytic known-answer tests (linear/quadratic fields, the x-ramp Laplacian of
// examples/main_3d_testing_grad.cpp:35-111, cosine-mode heat decay, exact
// conservation, Sod vs the exact Riemann solution) and by committed golden
// fixtures generated from it (tests/golden/make_golden.py).
//
// Arithmetic is written out operation by operation and compiled with
// -ffp-contract=off so that the FP64 GPU plain path (built with --fmad=false)
// reproduces it bit for bit.  Per-cell face sums run over face slots 0..5 in
// order, as the reference's device helper does
// (include/custom_cuda_functions.hpp:147-162).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

namespace fvo {

template <class R> struct V3 { R x, y, z; };
template <class R> inline V3<R> sub(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> add(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> inline R dot(V3<R> a, V3<R> b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
template <class R> inline R norm(V3<R> a) { return std::sqrt(dot(a, a)); }
template <class R> inline R csum(V3<R> a) { return (a.x + a.y) + a.z; }

// Face slots of a hexahedral cell: 0/1 = z-/z+, 2/3 = y-/y+, 4/5 = x-/x+
// (src/mesh3d.cpp:391-403); the opposite slot is f^1 (src/mesh3d.cpp:140-148).
inline int opposite(int f) { return f ^ 1; }

// Geometry in the reference's flattened N x 6 column-major form: entry (i, f)
// at f*n + i (include/decls.hpp:25-28, src/mesh3d.cpp:151-321).
template <class R> struct Mesh {
  int64_t nx = 0, ny = 0, nz = 0, n = 0;
  R dx = 0, dy = 0, dz = 0;
  std::vector<R> normal[3];      // "unsigned" normals (_normals)
  std::vector<R> normal_alt[3];  // outward unit normals (_normals_alt)
  std::vector<R> area, alpha_d, len_c2f;
  std::vector<R> volume, center[3], is_boundary;
  std::vector<int64_t> ids, ids_bound_free;

  int64_t cell(int64_t x, int64_t y, int64_t z) const { return nz * ny * x + nz * y + z; }
};

// Cell id = Z*Y*x + Z*y + z (src/mesh3d.cpp:387-389); vertex id likewise on the
// (X+1)(Y+1)(Z+1) lattice (src/mesh3d.cpp:405-416).
inline int64_t vertex_id(int64_t ny, int64_t nz, int64_t x, int64_t y, int64_t z) {
  return x * (nz + 1) * (ny + 1) + y * (nz + 1) + z;
}

// Vertex order of each face slot, as indices into the cell's 8 corner vertices
// v0..v7 = (x+a, y+b, z+c) with a,b,c in {0,1} ordered a-major
// (src/mesh3d.cpp:355-371).
static const int kFaceCorners[6][4] = {
    {0, 2, 6, 4}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 3, 7, 6}, {1, 3, 2, 0}, {5, 7, 6, 4}};

template <class R> struct FaceGeom { V3<R> normal, center; R area; };

// Geometry modes.  kGeomReference: Face3D::compute (src/mesh3d.cpp:43-62)
// with the norm of the half cross products as area; kGeomCompat: the same with
// the reference's component-sum area (exact only for axis-aligned faces,
// src/mesh3d.cpp:61); kGeomVectorArea (vertex meshes): the exact vector area
// S = (C - A) x (D - B) / 2 of the bilinear quad, n = S/|S|, A = |S|, and the
// cell volume taken about the cell centre -- with one-triangle normals and
// absolute coordinates the reference's volume formula turns negative on
// strongly jittered cells.  On axis-aligned faces all three agree.
enum { kGeomReference = 0, kGeomCompat = 1, kGeomVectorArea = 2 };

template <class R> FaceGeom<R> face_geom(const V3<R> c[4], int mode) {
  FaceGeom<R> g;
  V3<R> s{0, 0, 0};
  for (int i = 0; i < 4; ++i) s = add(s, c[i]);
  g.center = {s.x / R(4), s.y / R(4), s.z / R(4)};
  V3<R> AB = sub(c[1], c[0]), BC = sub(c[2], c[1]), CD = sub(c[3], c[2]);
  V3<R> AD = sub(c[3], c[0]), CB = sub(c[1], c[2]);
  if (mode == kGeomVectorArea) {
    V3<R> s2 = cross(sub(c[2], c[0]), sub(c[3], c[1]));
    V3<R> S{R(0.5) * s2.x, R(0.5) * s2.y, R(0.5) * s2.z};
    R len = norm(S);
    g.normal = {S.x / len, S.y / len, S.z / len};
    g.area = len;
    return g;
  }
  V3<R> nr = cross(AB, BC);
  R len = std::sqrt(dot(nr, nr));
  g.normal = {nr.x / len, nr.y / len, nr.z / len};
  V3<R> t1 = cross(AB, AD), t2 = cross(CB, CD);
  if (mode == kGeomCompat)
    g.area = R(0.5) * (std::fabs(csum(t1)) + std::fabs(csum(t2)));
  else
    g.area = R(0.5) * (norm(t1) + norm(t2));
  return g;
}

// Mesh3D::init_basic_internals + Mesh3D::compute (src/mesh3d.cpp:151-385),
// restated per cell.  verts: (X+1)(Y+1)(Z+1) x 3 coordinates in vertex-id
// order, or nullptr for the uniform lattice x*dx, y*dy, z*dz; mode is one of
// the geometry modes above.
template <class R>
void build_mesh(Mesh<R>& m, int64_t nx, int64_t ny, int64_t nz, double dx, double dy, double dz,
                const double* verts, int mode) {
  m.nx = nx; m.ny = ny; m.nz = nz; m.n = nx * ny * nz;
  m.dx = R(dx); m.dy = R(dy); m.dz = R(dz);
  const int64_t n = m.n;
  for (int d = 0; d < 3; ++d) {
    m.normal[d].assign(6 * n, 0); m.normal_alt[d].assign(6 * n, 0); m.center[d].assign(n, 0);
  }
  m.area.assign(6 * n, 0); m.alpha_d.assign(6 * n, 0); m.len_c2f.assign(6 * n, 0);
  m.volume.assign(n, 0); m.is_boundary.assign(n, 0);
  m.ids.assign(6 * n, 0); m.ids_bound_free.assign(6 * n, 0);

  auto vtx = [&](int64_t x, int64_t y, int64_t z) -> V3<R> {
    if (verts) {
      const double* p = verts + 3 * vertex_id(ny, nz, x, y, z);
      return {R(p[0]), R(p[1]), R(p[2])};
    }
    return {R(x) * m.dx, R(y) * m.dy, R(z) * m.dz};
  };
  auto corners = [&](int64_t x, int64_t y, int64_t z, V3<R> v[8]) {
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 2; ++c) v[a * 4 + b * 2 + c] = vtx(x + a, y + b, z + c);
  };
  auto cell_center = [&](const V3<R> v[8]) {
    V3<R> s{0, 0, 0};
    for (int i = 0; i < 8; ++i) s = add(s, v[i]);
    return V3<R>{s.x / R(8), s.y / R(8), s.z / R(8)};
  };

  // pass 1: cell centres
#pragma omp parallel for schedule(static)
  for (int64_t x = 0; x < nx; ++x)
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t z = 0; z < nz; ++z) {
        V3<R> v[8];
        corners(x, y, z, v);
        V3<R> c = cell_center(v);
        int64_t i = m.cell(x, y, z);
        m.center[0][i] = c.x; m.center[1][i] = c.y; m.center[2][i] = c.z;
      }

  // pass 2: per-cell faces (Quadrangle3D::compute, src/mesh3d.cpp:69-105) and
  // the N x 6 flattening (src/mesh3d.cpp:204-320)
#pragma omp parallel for schedule(static)
  for (int64_t x = 0; x < nx; ++x)
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t z = 0; z < nz; ++z) {
        const int64_t i = m.cell(x, y, z);
        V3<R> v[8];
        corners(x, y, z, v);
        const V3<R> cc{m.center[0][i], m.center[1][i], m.center[2][i]};
        R vol = 0;
        bool bnd = false;
        for (int f = 0; f < 6; ++f) {
          V3<R> fc[4];
          for (int k = 0; k < 4; ++k) fc[k] = v[kFaceCorners[f][k]];
          FaceGeom<R> g = face_geom(fc, mode);
          V3<R> good = dot(g.normal, sub(g.center, cc)) >= R(0)
                           ? g.normal : V3<R>{-g.normal.x, -g.normal.y, -g.normal.z};
          V3<R> uns = (f == 0 || f == 1 || f == 4 || f == 5)
                          ? V3<R>{-g.normal.x, -g.normal.y, -g.normal.z} : g.normal;
          const int64_t k6 = int64_t(f) * n + i;
          m.normal[0][k6] = uns.x; m.normal[1][k6] = uns.y; m.normal[2][k6] = uns.z;
          m.normal_alt[0][k6] = good.x; m.normal_alt[1][k6] = good.y; m.normal_alt[2][k6] = good.z;
          m.area[k6] = g.area;
          if (mode == kGeomVectorArea)
            vol = vol + dot(sub(g.center, cc), good) * g.area;
          else
            vol = vol + dot(g.center, good) * g.area;

          int64_t nbx = x, nby = y, nbz = z;
          if (f == 0) nbz = z - 1; else if (f == 1) nbz = z + 1;
          else if (f == 2) nby = y - 1; else if (f == 3) nby = y + 1;
          else if (f == 4) nbx = x - 1; else nbx = x + 1;
          const bool interior = nbx >= 0 && nbx < nx && nby >= 0 && nby < ny && nbz >= 0 && nbz < nz;
          V3<R> d;
          if (interior) {
            const int64_t j = m.cell(nbx, nby, nbz);
            m.ids[k6] = j; m.ids_bound_free[k6] = j;
            d = sub(V3<R>{m.center[0][j], m.center[1][j], m.center[2][j]}, cc);
          } else {
            bnd = true;
            m.ids[k6] = i; m.ids_bound_free[k6] = -1;
            d = sub(g.center, cc);
          }
          R cos_phi = dot(uns, d) / (norm(uns) * norm(d));
          R alpha = R(1) / cos_phi;
          m.alpha_d[k6] = interior ? std::fabs(alpha / norm(d)) : std::fabs(alpha / (norm(d) * R(2)));
          m.len_c2f[k6] = norm(sub(g.center, cc));
        }
        m.volume[i] = vol / R(3);
        m.is_boundary[i] = bnd ? R(1) : R(0);
      }
}

// ---------------------------------------------------------------------------
// Operators (reference operator layer).  Each has a per-cell form; the
// "faithful" CPU baseline runs the same arithmetic as full-array passes.
// ---------------------------------------------------------------------------

// GradVar: Green-Gauss gradient with linear face interpolation
// (src/fvm3d.cpp:808-823, include/grad_utils.hpp:23-36,82-99,
//  src/cuda_operators.cu:237-283).
template <class R> inline void grad_cell(const Mesh<R>& m, const R* phi, int64_t i, R g[3]) {
  const int64_t n = m.n;
  const R crr = phi[i];
  for (int d = 0; d < 3; ++d) {
    R acc = 0;
    for (int f = 0; f < 6; ++f) {
      const int64_t k6 = int64_t(f) * n + i;
      R itp = (crr + phi[m.ids[k6]]) * R(0.5);
      R t = itp * m.normal_alt[d][k6];
      acc = acc + t * m.area[k6];
    }
    g[d] = acc / m.volume[i];
  }
}

template <class R> void op_grad(const Mesh<R>& m, const R* phi, R* out, int mask) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i) {
    R g[3];
    grad_cell(m, phi, i, g);
    R acc = 0;
    for (int d = 0; d < 3; ++d) if (mask & (1 << d)) acc = acc + g[d];
    out[i] = acc;
  }
}

// Grad2Var: orthogonal Laplacian, (phi_N - phi_P) * alpha_d summed with the
// unsigned normals (src/fvm3d.cpp:880-900, include/grad_utils.hpp:101-125,
// src/cuda_operators.cu:490-544).  Boundary faces see phi_N = phi_P.
template <class R> inline R lapl_cell(const Mesh<R>& m, const R* phi, int64_t i, int mask) {
  const int64_t n = m.n;
  const R crr = phi[i];
  R sn[6];
  for (int f = 0; f < 6; ++f) {
    const int64_t k6 = int64_t(f) * n + i;
    sn[f] = (phi[m.ids[k6]] - crr) * m.alpha_d[k6];
  }
  R res = 0;
  for (int d = 0; d < 3; ++d) {
    if (!(mask & (1 << d))) continue;
    R acc = 0;
    for (int f = 0; f < 6; ++f) {
      const int64_t k6 = int64_t(f) * n + i;
      R t = sn[f] * m.normal[d][k6];
      acc = acc + t * m.area[k6];
    }
    res = res + acc / m.volume[i];
  }
  return res;
}

template <class R> void op_lapl(const Mesh<R>& m, const R* phi, R* out, int mask) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i) out[i] = lapl_cell(m, phi, i, mask);
}

// StabVar: upwind face extrapolation phi + |x_f - x_P| g_d n_alt, then half the
// jump against the neighbour's opposite-face value, summed with the unsigned
// normals (src/fvm3d.cpp:915-936, include/grad_utils.hpp:38-80,
// src/cuda_operators.cu:307-434).  A boundary face reads the cell's own
// opposite-face value, as the reference does.
template <class R> void op_stab(const Mesh<R>& m, const R* phi, R* out, int mask) {
  const int64_t n = m.n;
  std::vector<R> up(3 * 6 * n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    R g[3];
    grad_cell(m, phi, i, g);
    for (int d = 0; d < 3; ++d)
      for (int f = 0; f < 6; ++f) {
        const int64_t k6 = int64_t(f) * n + i;
        up[int64_t(d) * 6 * n + k6] = phi[i] + m.len_c2f[k6] * g[d] * m.normal_alt[d][k6];
      }
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    R res = 0;
    for (int d = 0; d < 3; ++d) {
      if (!(mask & (1 << d))) continue;
      const R* u = up.data() + int64_t(d) * 6 * n;
      R acc = 0;
      for (int f = 0; f < 6; ++f) {
        const int64_t k6 = int64_t(f) * n + i;
        R col = u[int64_t(opposite(f)) * n + m.ids[k6]];
        R s = R(0.5) * (u[k6] - col);
        R t = s * m.normal[d][k6];
        acc = acc + t * m.area[k6];
      }
      res = res + acc / m.volume[i];
    }
    out[i] = res;
  }
}

// DtVar / D2tVar updates (src/fvm3d.cpp:690-692, 735-740): forward Euler and
// the leapfrog second-order update, operation order as in the CPU extract.
template <class R> inline R d1t_update(R rhs, R cur, R dt) { return dt * rhs + cur; }
template <class R> inline R d2t_update(R rhs, R cur, R prev, R dt) { return (dt * dt * rhs + R(2) * cur) - prev; }

// UpdatePolicies::CourantFriedrichsLewy3D / 1D (src/fvm3d.cpp:512-556):
// dt = CFL * min_P dl / (sqrt(gamma p / rho) + |u|).
template <class R>
R cfl_reference(const Mesh<R>& m, R cfl, R gamma, const R* p, const R* rho, const R* u, const R* v,
                const R* w) {
  R dl = std::min(std::min(m.dx, m.dy), m.dz);
  R best = INFINITY;
  for (int64_t i = 0; i < m.n; ++i) {
    R vv = u[i] * u[i];
    if (v) vv = vv + v[i] * v[i];
    if (w) vv = vv + w[i] * w[i];
    R den = dl * (R(1) / (std::sqrt((gamma * p[i]) / rho[i]) + std::sqrt(vv)));
    best = std::min(best, den);
  }
  return cfl * best;
}

// Heat equation d1t(T) = k * lapl(T) with the zero-gradient boundary intrinsic
// to Grad2Var (examples/main_3d_heat.cpp:89-91): per step L = lapl(T),
// R = k * L, T' = dt * R + T.
template <class R> void heat_step(const Mesh<R>& m, const R* T, R* Tn, R k, R dt) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i) {
    R L = lapl_cell(m, T, i, 7);
    R rhs = k * L;
    Tn[i] = d1t_update(rhs, T[i], dt);
  }
}

// Faithful (Eigen-like, full-array passes) heat step used as the timed CPU
// baseline: the same arithmetic as heat_step through N x 6 temporaries.
template <class R> void heat_step_faithful(const Mesh<R>& m, const R* T, R* Tn, R k, R dt, std::vector<R>& tmp) {
  const int64_t n = m.n;
  tmp.resize(7 * n);
  R* sn = tmp.data();
  R* L = tmp.data() + 6 * n;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i)
    for (int f = 0; f < 6; ++f) {
      const int64_t k6 = int64_t(f) * n + i;
      sn[k6] = (T[m.ids[k6]] - T[i]) * m.alpha_d[k6];
    }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    R res = 0;
    for (int d = 0; d < 3; ++d) {
      R acc = 0;
      for (int f = 0; f < 6; ++f) {
        const int64_t k6 = int64_t(f) * n + i;
        R t = sn[k6] * m.normal[d][k6];
        acc = acc + t * m.area[k6];
      }
      res = res + acc / m.volume[i];
    }
    L[i] = res;
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) Tn[i] = d1t_update(k * L[i], T[i], dt);
}

// ---------------------------------------------------------------------------
// First-order acoustic system (p, u, v, w), rho = 1:
//   p_t = -c^2 div(u),  u_t = -grad(p)
// Rusanov flux per face with outward unit normal nh and area A:
//   F_p = c_P^2 * 0.5 (un_P + un_N) - 0.5 c_f (p_N - p_P)
//   F_u = 0.5 (p_P + p_N) nh       - 0.5 c_f (u_N - u_P)
// R = -(1/V) sum_f F A; q' = q + dt R.  Reflective wall: ghost p = p_P,
// u_G = u_P - 2 (u_P . nh) nh, c_G = c_P.  c_f = max(c_P, c_N) (speed_mode 0)
// or 0.5 (c_P + c_N) (speed_mode 1, the differentiable choice).
// State layout: q = [p | u | v | w], each block n values.
// ---------------------------------------------------------------------------
template <class R>
inline void wave_rhs_cell(const Mesh<R>& m, const R* q, const R* cfield, R cconst, int speed_mode, int64_t i,
                          R out[4]) {
  const int64_t n = m.n;
  const R pP = q[i], uP = q[n + i], vP = q[2 * n + i], wP = q[3 * n + i];
  const R cP = cfield ? cfield[i] : cconst;
  const R c2 = cP * cP;
  R ap = 0, au = 0, av = 0, aw = 0;
  for (int f = 0; f < 6; ++f) {
    const int64_t k6 = int64_t(f) * n + i;
    const R nx = m.normal_alt[0][k6], ny = m.normal_alt[1][k6], nz = m.normal_alt[2][k6];
    const R A = m.area[k6];
    const R unP = (uP * nx + vP * ny) + wP * nz;
    R pN, uN, vN, wN, cN;
    if (m.ids_bound_free[k6] >= 0) {
      const int64_t j = m.ids[k6];
      pN = q[j]; uN = q[n + j]; vN = q[2 * n + j]; wN = q[3 * n + j];
      cN = cfield ? cfield[j] : cconst;
    } else {
      const R two_un = R(2) * unP;
      pN = pP; uN = uP - two_un * nx; vN = vP - two_un * ny; wN = wP - two_un * nz; cN = cP;
    }
    const R unN = (uN * nx + vN * ny) + wN * nz;
    const R cf = speed_mode == 0 ? std::max(cP, cN) : R(0.5) * (cP + cN);
    const R hc = R(0.5) * cf;
    const R fp = c2 * (R(0.5) * (unP + unN)) - hc * (pN - pP);
    const R pm = R(0.5) * (pP + pN);
    const R fu = pm * nx - hc * (uN - uP);
    const R fv = pm * ny - hc * (vN - vP);
    const R fw = pm * nz - hc * (wN - wP);
    ap = ap + fp * A; au = au + fu * A; av = av + fv * A; aw = aw + fw * A;
  }
  const R V = m.volume[i];
  out[0] = -(ap / V); out[1] = -(au / V); out[2] = -(av / V); out[3] = -(aw / V);
}

template <class R>
void wave_step(const Mesh<R>& m, const R* q, R* qn, const R* cfield, R cconst, int speed_mode, R dt) {
  const int64_t n = m.n;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    R r[4];
    wave_rhs_cell(m, q, cfield, cconst, speed_mode, i, r);
    for (int c = 0; c < 4; ++c) qn[int64_t(c) * n + i] = d1t_update(r[c], q[int64_t(c) * n + i], dt);
  }
}

// Faithful (full-array) wave step used as the CPU baseline: face states are
// gathered into N x 6 temporaries first, then fluxes, then the reduction, the
// way an operator-by-operator Eigen evaluation would stream them.
template <class R>
void wave_step_faithful(const Mesh<R>& m, const R* q, R* qn, R cconst, R dt, std::vector<R>& tmp) {
  const int64_t n = m.n;
  tmp.resize(4 * 6 * n);
  R* nb[4] = {tmp.data(), tmp.data() + 6 * n, tmp.data() + 12 * n, tmp.data() + 18 * n};
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i)
    for (int f = 0; f < 6; ++f) {
      const int64_t k6 = int64_t(f) * n + i;
      const int64_t j = m.ids[k6];
      for (int c = 0; c < 4; ++c) nb[c][k6] = q[int64_t(c) * n + j];
      if (m.ids_bound_free[k6] < 0) {
        const R nx = m.normal_alt[0][k6], ny = m.normal_alt[1][k6], nz = m.normal_alt[2][k6];
        const R two_un = R(2) * ((q[n + i] * nx + q[2 * n + i] * ny) + q[3 * n + i] * nz);
        nb[1][k6] = q[n + i] - two_un * nx; nb[2][k6] = q[2 * n + i] - two_un * ny;
        nb[3][k6] = q[3 * n + i] - two_un * nz;
      }
    }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const R pP = q[i], uP = q[n + i], vP = q[2 * n + i], wP = q[3 * n + i];
    const R c2 = cconst * cconst, hc = R(0.5) * cconst;
    R ap = 0, au = 0, av = 0, aw = 0;
    for (int f = 0; f < 6; ++f) {
      const int64_t k6 = int64_t(f) * n + i;
      const R nx = m.normal_alt[0][k6], ny = m.normal_alt[1][k6], nz = m.normal_alt[2][k6];
      const R A = m.area[k6];
      const R unP = (uP * nx + vP * ny) + wP * nz;
      const R pN = nb[0][k6], uN = nb[1][k6], vN = nb[2][k6], wN = nb[3][k6];
      const R unN = (uN * nx + vN * ny) + wN * nz;
      const R fp = c2 * (R(0.5) * (unP + unN)) - hc * (pN - pP);
      const R pm = R(0.5) * (pP + pN);
      ap = ap + fp * A;
      au = au + (pm * nx - hc * (uN - uP)) * A;
      av = av + (pm * ny - hc * (vN - vP)) * A;
      aw = aw + (pm * nz - hc * (wN - wP)) * A;
    }
    const R V = m.volume[i];
    qn[i] = d1t_update(-(ap / V), pP, dt);
    qn[n + i] = d1t_update(-(au / V), uP, dt);
    qn[2 * n + i] = d1t_update(-(av / V), vP, dt);
    qn[3 * n + i] = d1t_update(-(aw / V), wP, dt);
  }
}

// dt for the wave system: CFL * min_P 2 V_P / sum_f c_P A_f.  On a uniform mesh
// this equals CFL / sum_d (c / dx_d).
template <class R> double wave_dt(const Mesh<R>& m, const R* cfield, double cconst, double cfl) {
  double best = INFINITY;
  for (int64_t i = 0; i < m.n; ++i) {
    double c = cfield ? double(cfield[i]) : cconst;
    double s = 0;
    for (int f = 0; f < 6; ++f) s += c * double(m.area[int64_t(f) * m.n + i]);
    best = std::min(best, 2.0 * double(m.volume[i]) / s);
  }
  return cfl * best;
}

// ---------------------------------------------------------------------------
// Adjoint of the wave step for speed_mode 1 (c_f = (c_P + c_N)/2).  With
// q' = q + dt A(c) q:  lam = lam' + dt A^T lam',
// g_c += dt (d(A q)/dc)^T lam'.  A^T is applied as a gather over the 6
// neighbours (the transpose of the flux scatter).
// ---------------------------------------------------------------------------
template <class R>
void wave_adjoint_step(const Mesh<R>& m, const R* q, const R* lam1, R* lam0, const R* cf, R* gc, R dt) {
  const int64_t n = m.n;
  // Volume-scaled adjoint lt = lam / V lets neighbour terms carry their own
  // cell volume (R(N) holds 1/V_N).
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const R cP = cf[i];
    const R iVP = R(1) / m.volume[i];
    const R lpP = lam1[i] * iVP, luP = lam1[n + i] * iVP, lvP = lam1[2 * n + i] * iVP, lwP = lam1[3 * n + i] * iVP;
    const R pP = q[i], uP = q[n + i], vP = q[2 * n + i], wP = q[3 * n + i];
    R ap = 0, au = 0, av = 0, aw = 0, g = 0;
    for (int f = 0; f < 6; ++f) {
      const int64_t k6 = int64_t(f) * n + i;
      const R nx = m.normal_alt[0][k6], ny = m.normal_alt[1][k6], nz = m.normal_alt[2][k6];
      const R A = m.area[k6];
      const R Sx = nx * A, Sy = ny * A, Sz = nz * A;
      if (m.ids_bound_free[k6] >= 0) {
        const int64_t j = m.ids[k6];
        const R cN = cf[j];
        const R iVN = R(1) / m.volume[j];
        const R h = R(0.5) * (R(0.5) * (cP + cN)) * A;  // c_f A / 2
        const R lpN = lam1[j] * iVN, luN = lam1[n + j] * iVN, lvN = lam1[2 * n + j] * iVN, lwN = lam1[3 * n + j] * iVN;
        // (A^T lam)_p: (c_f A/2)(lt_pN - lt_pP) + (1/2) S.(lt_uN - lt_uP)
        const R Slu_d = (Sx * (luN - luP) + Sy * (lvN - lvP)) + Sz * (lwN - lwP);
        ap = ap + (h * (lpN - lpP) + R(0.5) * Slu_d);
        // (A^T lam)_u: (1/2) S (c_N^2 lt_pN - c_P^2 lt_pP) + (c_f A/2)(lt_uN - lt_uP)
        const R sp = R(0.5) * (cN * cN * lpN - cP * cP * lpP);
        au = au + (sp * Sx + h * (luN - luP));
        av = av + (sp * Sy + h * (lvN - lvP));
        aw = aw + (sp * Sz + h * (lwN - lwP));
        // d/dc_P: the c_P^2 term of R_p(P) and c_f = (c_P + c_N)/2 in R(P), R(N)
        const R pN = q[j], uN = q[n + j], vN = q[2 * n + j], wN = q[3 * n + j];
        const R Su_sum = (Sx * (uP + uN) + Sy * (vP + vN)) + Sz * (wP + wN);
        g = g - cP * Su_sum * lpP;
        const R jp = pN - pP;
        const R ju_self = ((uN - uP) * luP + (vN - vP) * lvP) + (wN - wP) * lwP;
        const R ju_nb = ((uP - uN) * luN + (vP - vN) * lvN) + (wP - wN) * lwN;
        g = g + R(0.25) * A * ((jp * lpP + ju_self) + (ju_nb - jp * lpN));
      } else {
        // reflective wall: R_p gets nothing; R_u gets -(p_P S + c_P A (u_P.nh) nh)/V
        const R Slu = (Sx * luP + Sy * lvP) + Sz * lwP;
        ap = ap - Slu;
        const R lun = (luP * nx + lvP * ny) + lwP * nz;
        const R cA = cP * A;
        au = au - cA * lun * nx; av = av - cA * lun * ny; aw = aw - cA * lun * nz;
        const R un = (uP * nx + vP * ny) + wP * nz;
        g = g - A * un * lun;
      }
    }
    lam0[i] = lam1[i] + dt * ap;
    lam0[n + i] = lam1[n + i] + dt * au;
    lam0[2 * n + i] = lam1[2 * n + i] + dt * av;
    lam0[3 * n + i] = lam1[3 * n + i] + dt * aw;
    gc[i] = gc[i] + dt * g;
  }
}

// ---------------------------------------------------------------------------
// Compressible Euler, first-order Rusanov, conserved U = [rho|mx|my|mz|E].
// Faces in slots 4/5 (x ends) are zero-gradient (ghost = U_P); the other
// boundary faces are reflective walls (normal momentum flipped).
// ---------------------------------------------------------------------------
template <class R> struct EulerPrim { R rho, u, v, w, p, a; };

template <class R> inline EulerPrim<R> euler_prim(R rho, R mx, R my, R mz, R E, R gamma) {
  EulerPrim<R> s;
  s.rho = rho;
  s.u = mx / rho; s.v = my / rho; s.w = mz / rho;
  const R ke = R(0.5) * ((mx * s.u + my * s.v) + mz * s.w);
  s.p = (gamma - R(1)) * (E - ke);
  s.a = std::sqrt(gamma * s.p / rho);
  return s;
}

template <class R>
inline void euler_rhs_cell(const Mesh<R>& m, const R* U, R gamma, int64_t i, R out[5]) {
  const int64_t n = m.n;
  const R rP = U[i], mxP = U[n + i], myP = U[2 * n + i], mzP = U[3 * n + i], EP = U[4 * n + i];
  const EulerPrim<R> P = euler_prim(rP, mxP, myP, mzP, EP, gamma);
  R acc[5] = {0, 0, 0, 0, 0};
  for (int f = 0; f < 6; ++f) {
    const int64_t k6 = int64_t(f) * n + i;
    const R nx = m.normal_alt[0][k6], ny = m.normal_alt[1][k6], nz = m.normal_alt[2][k6];
    const R A = m.area[k6];
    R rN, mxN, myN, mzN, EN;
    if (m.ids_bound_free[k6] >= 0) {
      const int64_t j = m.ids[k6];
      rN = U[j]; mxN = U[n + j]; myN = U[2 * n + j]; mzN = U[3 * n + j]; EN = U[4 * n + j];
    } else if (f >= 4) {
      rN = rP; mxN = mxP; myN = myP; mzN = mzP; EN = EP;
    } else {
      const R two_mn = R(2) * ((mxP * nx + myP * ny) + mzP * nz);
      rN = rP; mxN = mxP - two_mn * nx; myN = myP - two_mn * ny; mzN = mzP - two_mn * nz; EN = EP;
    }
    const EulerPrim<R> N = euler_prim(rN, mxN, myN, mzN, EN, gamma);
    const R unP = (P.u * nx + P.v * ny) + P.w * nz;
    const R unN = (N.u * nx + N.v * ny) + N.w * nz;
    const R lam = std::max(std::fabs(unP) + P.a, std::fabs(unN) + N.a);
    const R hl = R(0.5) * lam;
    const R f0 = R(0.5) * (rP * unP + rN * unN) - hl * (rN - rP);
    const R f1 = R(0.5) * ((mxP * unP + P.p * nx) + (mxN * unN + N.p * nx)) - hl * (mxN - mxP);
    const R f2 = R(0.5) * ((myP * unP + P.p * ny) + (myN * unN + N.p * ny)) - hl * (myN - myP);
    const R f3 = R(0.5) * ((mzP * unP + P.p * nz) + (mzN * unN + N.p * nz)) - hl * (mzN - mzP);
    const R f4 = R(0.5) * ((EP + P.p) * unP + (EN + N.p) * unN) - hl * (EN - EP);
    acc[0] = acc[0] + f0 * A; acc[1] = acc[1] + f1 * A; acc[2] = acc[2] + f2 * A;
    acc[3] = acc[3] + f3 * A; acc[4] = acc[4] + f4 * A;
  }
  const R V = m.volume[i];
  for (int c = 0; c < 5; ++c) out[c] = -(acc[c] / V);
}

// Per-direction maximum signal speed max_P |u_d| + a.
template <class R> void euler_max_speeds(const Mesh<R>& m, const R* U, R gamma, R lam[3]) {
  const int64_t n = m.n;
  lam[0] = lam[1] = lam[2] = 0;
  for (int64_t i = 0; i < n; ++i) {
    EulerPrim<R> s = euler_prim(U[i], U[n + i], U[2 * n + i], U[3 * n + i], U[4 * n + i], gamma);
    lam[0] = std::max(lam[0], std::fabs(s.u) + s.a);
    lam[1] = std::max(lam[1], std::fabs(s.v) + s.a);
    lam[2] = std::max(lam[2], std::fabs(s.w) + s.a);
  }
}

template <class R> void euler_step(const Mesh<R>& m, const R* U, R* Un, R gamma, R dt) {
  const int64_t n = m.n;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    R r[5];
    euler_rhs_cell(m, U, gamma, i, r);
    for (int c = 0; c < 5; ++c) Un[int64_t(c) * n + i] = d1t_update(r[c], U[int64_t(c) * n + i], dt);
  }
}

// Neumaier-compensated sum of field * V in double.
template <class R> double neumaier_total(const Mesh<R>& m, const R* f) {
  double s = 0, c = 0;
  for (int64_t i = 0; i < m.n; ++i) {
    double x = double(f[i]) * double(m.volume[i]);
    double t = s + x;
    if (std::fabs(s) >= std::fabs(x)) c += (s - t) + x; else c += (x - t) + s;
    s = t;
  }
  return s + c;
}

}  // namespace fvo
