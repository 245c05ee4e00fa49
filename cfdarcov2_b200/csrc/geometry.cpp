// Host geometry of the hexahedral mesh, following the reference's
// Mesh3D::init_basic_internals / Face3D::compute / Quadrangle3D::compute /
// Mesh3D::compute (src/mesh3d.cpp:43-385).  Built in double with every
// multiply and add separately rounded (compiled with -ffp-contract=off) so the
// FP64 plain kernels see exactly the arrays the CPU oracle restates.
//
// Differences from the reference, on purpose:
//  * computed per cell in one pass instead of through shared_ptr object graphs
//    (same formulas and operation order; a shared face is computed by both
//    cells from the same vertex order, so both see identical values);
//  * uniform lattices use the reference formulas with the norm of the two
//    half cross products as face area (the reference's component sum,
//    src/mesh3d.cpp:61, is identical on axis-aligned faces);
//  * vertex meshes default to the exact vector area of each bilinear face,
//    S = (C - A) x (D - B) / 2 (n = S/|S|, A = |S|), and a volume taken about
//    the cell centre: with one-triangle normals and absolute coordinates the
//    reference's volume formula goes negative on strongly jittered cells.
//    CFDB_MESH_COMPAT_AREA restores the reference formulas verbatim;
//  * the unused _n_min_alpha_d arrays (non-orthogonal correction, commented
//    out in include/grad_utils.hpp:117-122) are not built.
#include <cmath>
#include <new>

#include "cfdb_internal.hpp"

namespace {

struct P3 { double x, y, z; };
inline P3 sub(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline P3 add(P3 a, P3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline P3 neg(P3 a) { return {-a.x, -a.y, -a.z}; }
inline P3 cross(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double dot(P3 a, P3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline double nrm(P3 a) { return std::sqrt(dot(a, a)); }
inline double csum(P3 a) { return (a.x + a.y) + a.z; }

// Corner k of a cell is (x+a, y+b, z+c) with k = 4a + 2b + c; each face slot
// lists its four corners in the reference's order (src/mesh3d.cpp:355-371).
const int kCorners[6][4] = {{0, 2, 6, 4}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 3, 7, 6}, {1, 3, 2, 0}, {5, 7, 6, 4}};

struct Face { P3 normal, center; double area; };

enum { kGeomReference = 0, kGeomCompat = 1, kGeomVectorArea = 2 };

Face face_of(const P3 c[4], int mode) {
  Face f;
  P3 s{0, 0, 0};
  for (int i = 0; i < 4; ++i) s = add(s, c[i]);
  f.center = {s.x / 4.0, s.y / 4.0, s.z / 4.0};
  if (mode == kGeomVectorArea) {
    const P3 s2 = cross(sub(c[2], c[0]), sub(c[3], c[1]));
    const P3 S{0.5 * s2.x, 0.5 * s2.y, 0.5 * s2.z};
    const double len = nrm(S);
    f.normal = {S.x / len, S.y / len, S.z / len};
    f.area = len;
    return f;
  }
  const P3 AB = sub(c[1], c[0]), BC = sub(c[2], c[1]), CD = sub(c[3], c[2]);
  const P3 AD = sub(c[3], c[0]), CB = sub(c[1], c[2]);
  const P3 nr = cross(AB, BC);
  const double len = std::sqrt(dot(nr, nr));
  f.normal = {nr.x / len, nr.y / len, nr.z / len};
  const P3 t1 = cross(AB, AD), t2 = cross(CB, CD);
  f.area = mode == kGeomCompat ? 0.5 * (std::fabs(csum(t1)) + std::fabs(csum(t2))) : 0.5 * (nrm(t1) + nrm(t2));
  return f;
}

}  // namespace

bool cfdb_build_geometry(HostGeom& g, int64_t nx, int64_t ny, int64_t nz, double dx, double dy, double dz,
                         const double* verts, int mode) {
  const int64_t n = nx * ny * nz;
  g.nx = nx; g.ny = ny; g.nz = nz; g.n = n;
  try {
    g.normal.assign(18 * n, 0.0); g.normal_alt.assign(18 * n, 0.0);
    g.area.assign(6 * n, 0.0); g.alpha.assign(6 * n, 0.0); g.len.assign(6 * n, 0.0);
    g.volume.assign(n, 0.0); g.center.assign(3 * n, 0.0); g.isb.assign(n, 0.0);
    g.ids.assign(6 * n, 0); g.ibf.assign(6 * n, 0);
  } catch (const std::bad_alloc&) {
    return false;
  }
  auto cell_id = [&](int64_t x, int64_t y, int64_t z) { return nz * ny * x + nz * y + z; };
  auto vtx = [&](int64_t x, int64_t y, int64_t z) -> P3 {
    if (verts) {
      const double* p = verts + 3 * (x * (nz + 1) * (ny + 1) + y * (nz + 1) + z);
      return {p[0], p[1], p[2]};
    }
    return {double(x) * dx, double(y) * dy, double(z) * dz};
  };
  auto corners = [&](int64_t x, int64_t y, int64_t z, P3 v[8]) {
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 2; ++c) v[a * 4 + b * 2 + c] = vtx(x + a, y + b, z + c);
  };

#pragma omp parallel for schedule(static)
  for (int64_t x = 0; x < nx; ++x)
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t z = 0; z < nz; ++z) {
        P3 v[8];
        corners(x, y, z, v);
        P3 s{0, 0, 0};
        for (int k = 0; k < 8; ++k) s = add(s, v[k]);
        const int64_t i = cell_id(x, y, z);
        g.center[i] = s.x / 8.0; g.center[n + i] = s.y / 8.0; g.center[2 * n + i] = s.z / 8.0;
      }

#pragma omp parallel for schedule(static)
  for (int64_t x = 0; x < nx; ++x)
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t z = 0; z < nz; ++z) {
        const int64_t i = cell_id(x, y, z);
        P3 v[8];
        corners(x, y, z, v);
        const P3 cc{g.center[i], g.center[n + i], g.center[2 * n + i]};
        double vol = 0.0;
        bool bnd = false;
        for (int f = 0; f < 6; ++f) {
          P3 fc[4];
          for (int k = 0; k < 4; ++k) fc[k] = v[kCorners[f][k]];
          const Face fg = face_of(fc, mode);
          const P3 good = dot(fg.normal, sub(fg.center, cc)) >= 0.0 ? fg.normal : neg(fg.normal);
          const P3 uns = (f == 0 || f == 1 || f == 4 || f == 5) ? neg(fg.normal) : fg.normal;
          const int64_t k6 = int64_t(f) * n + i;
          g.normal[k6] = uns.x; g.normal[6 * n + k6] = uns.y; g.normal[12 * n + k6] = uns.z;
          g.normal_alt[k6] = good.x; g.normal_alt[6 * n + k6] = good.y; g.normal_alt[12 * n + k6] = good.z;
          g.area[k6] = fg.area;
          vol = vol + dot(mode == kGeomVectorArea ? sub(fg.center, cc) : fg.center, good) * fg.area;

          int64_t bx = x, by = y, bz = z;
          switch (f) {
            case 0: bz = z - 1; break;
            case 1: bz = z + 1; break;
            case 2: by = y - 1; break;
            case 3: by = y + 1; break;
            case 4: bx = x - 1; break;
            default: bx = x + 1; break;
          }
          const bool interior = bx >= 0 && bx < nx && by >= 0 && by < ny && bz >= 0 && bz < nz;
          P3 d;
          if (interior) {
            const int64_t j = cell_id(bx, by, bz);
            g.ids[k6] = j; g.ibf[k6] = j;
            d = sub(P3{g.center[j], g.center[n + j], g.center[2 * n + j]}, cc);
          } else {
            bnd = true;
            g.ids[k6] = i; g.ibf[k6] = -1;
            d = sub(fg.center, cc);
          }
          const double cos_phi = dot(uns, d) / (nrm(uns) * nrm(d));
          const double alpha = 1.0 / cos_phi;
          g.alpha[k6] = interior ? std::fabs(alpha / nrm(d)) : std::fabs(alpha / (nrm(d) * 2.0));
          g.len[k6] = nrm(sub(fg.center, cc));
        }
        g.volume[i] = vol / 3.0;
        g.isb[i] = bnd ? 1.0 : 0.0;
      }
  return true;
}
