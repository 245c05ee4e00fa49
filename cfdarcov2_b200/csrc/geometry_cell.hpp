// Per-cell geometry of the hexahedral mesh, shared by the host builder
// (geometry.cpp, compiled with -ffp-contract=off) and the device builder
// (geometry_dev.cu, compiled with --fmad=false and IEEE division and square
// root).  Every multiply, add, divide and square root is separately rounded
// on both sides, so the two builders produce the same doubles bit for bit.
//
// Formulas follow the reference's Mesh3D::init_basic_internals /
// Face3D::compute / Quadrangle3D::compute / Mesh3D::compute
// (src/mesh3d.cpp:43-385); the differences on purpose are listed in
// geometry.cpp.
#pragma once
#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define CFDB_HD __host__ __device__ __forceinline__
#else
#define CFDB_HD inline
#endif

namespace cfdb_geom {

struct P3 { double x, y, z; };
CFDB_HD P3 sub(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
CFDB_HD P3 add(P3 a, P3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
CFDB_HD P3 neg(P3 a) { return {-a.x, -a.y, -a.z}; }
CFDB_HD P3 cross(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
CFDB_HD double dot(P3 a, P3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
CFDB_HD double nrm(P3 a) { return sqrt(dot(a, a)); }
CFDB_HD double csum(P3 a) { return (a.x + a.y) + a.z; }

enum { kGeomReference = 0, kGeomCompat = 1, kGeomVectorArea = 2 };

// Corner k of a cell is (x+a, y+b, z+c) with k = 4a + 2b + c; face slot f
// lists its four corners in the reference's order (src/mesh3d.cpp:355-371).
CFDB_HD int corner(int f, int k) {
  const int c[6][4] = {{0, 2, 6, 4}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 3, 7, 6}, {1, 3, 2, 0}, {5, 7, 6, 4}};
  return c[f][k];
}

struct Face { P3 normal, center; double area; };

CFDB_HD Face face_of(const P3 c[4], int mode) {
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
  const double len = sqrt(dot(nr, nr));
  f.normal = {nr.x / len, nr.y / len, nr.z / len};
  const P3 t1 = cross(AB, AD), t2 = cross(CB, CD);
  f.area = mode == kGeomCompat ? 0.5 * (fabs(csum(t1)) + fabs(csum(t2))) : 0.5 * (nrm(t1) + nrm(t2));
  return f;
}

// Vertex (x, y, z) of the lattice: x dx, y dy, z dz, or the vertex array
// (x-major, (nx+1)(ny+1)(nz+1) points of 3 doubles).
struct Lattice {
  int64_t nx, ny, nz;
  double dx, dy, dz;
  const double* verts;  // null: uniform lattice
  CFDB_HD P3 vtx(int64_t x, int64_t y, int64_t z) const {
    if (verts) {
      const double* p = verts + 3 * (x * (nz + 1) * (ny + 1) + y * (nz + 1) + z);
      return {p[0], p[1], p[2]};
    }
    return {double(x) * dx, double(y) * dy, double(z) * dz};
  }
  CFDB_HD void corners(int64_t x, int64_t y, int64_t z, P3 v[8]) const {
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 2; ++c) v[a * 4 + b * 2 + c] = vtx(x + a, y + b, z + c);
  }
  CFDB_HD int64_t id(int64_t x, int64_t y, int64_t z) const { return nz * ny * x + nz * y + z; }
  // cell centre: the mean of the eight corners, summed in corner order
  CFDB_HD P3 center(int64_t x, int64_t y, int64_t z) const {
    P3 v[8];
    corners(x, y, z, v);
    P3 s{0, 0, 0};
    for (int k = 0; k < 8; ++k) s = add(s, v[k]);
    return {s.x / 8.0, s.y / 8.0, s.z / 8.0};
  }
};

// The geometry of face slot f of one cell.
struct CellFace {
  P3 uns, good;   // the reference's unsigned normal and the outward normal
  double area, alpha, len;
  int64_t id, ibf;  // neighbour (the cell itself on a wall) and -1 on a wall
};

// Computes the six faces of cell (x, y, z), handing each to face(f, o) as
// it is done (no per-cell face array: the device builders keep one face in
// registers), and returns the cell's volume; *boundary is set when a face
// lies on the wall.  center_of(x, y, z) gives a cell centre (the same value
// Lattice::center computes).
template <class CenterOf, class FaceSink>
CFDB_HD double cell_geometry(const Lattice& L, int64_t x, int64_t y, int64_t z, int mode, CenterOf center_of,
                             FaceSink face, bool* boundary) {
  const int64_t i = L.id(x, y, z);
  P3 v[8];
  L.corners(x, y, z, v);
  const P3 cc = center_of(x, y, z);
  double vol = 0.0;
  bool bnd = false;
  for (int f = 0; f < 6; ++f) {
    P3 fc[4];
    for (int k = 0; k < 4; ++k) fc[k] = v[corner(f, k)];
    const Face fg = face_of(fc, mode);
    const P3 good = dot(fg.normal, sub(fg.center, cc)) >= 0.0 ? fg.normal : neg(fg.normal);
    const P3 uns = (f == 0 || f == 1 || f == 4 || f == 5) ? neg(fg.normal) : fg.normal;
    CellFace o;
    o.uns = uns;
    o.good = good;
    o.area = fg.area;
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
    const bool interior = bx >= 0 && bx < L.nx && by >= 0 && by < L.ny && bz >= 0 && bz < L.nz;
    P3 d;
    if (interior) {
      const int64_t j = L.id(bx, by, bz);
      o.id = j;
      o.ibf = j;
      d = sub(center_of(bx, by, bz), cc);
    } else {
      bnd = true;
      o.id = i;
      o.ibf = -1;
      d = sub(fg.center, cc);
    }
    const double cos_phi = dot(uns, d) / (nrm(uns) * nrm(d));
    const double alpha = 1.0 / cos_phi;
    o.alpha = interior ? fabs(alpha / nrm(d)) : fabs(alpha / (nrm(d) * 2.0));
    o.len = nrm(sub(fg.center, cc));
    face(f, o);
  }
  *boundary = bnd;
  return vol / 3.0;
}

}  // namespace cfdb_geom
