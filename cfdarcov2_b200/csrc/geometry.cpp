// Host geometry of the hexahedral mesh, following the reference's
// Mesh3D::init_basic_internals / Face3D::compute / Quadrangle3D::compute /
// Mesh3D::compute (src/mesh3d.cpp:43-385).  Built in double with every
// multiply and add separately rounded (compiled with -ffp-contract=off) so the
// FP64 plain kernels see exactly the arrays the CPU oracle restates.  The
// per-cell formulas live in geometry_cell.hpp, shared with the device
// builder (geometry_dev.cu) that gives the same doubles.
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
#include <new>

#include "cfdb_internal.hpp"
#include "geometry_cell.hpp"

bool cfdb_build_geometry(HostGeom& g, int64_t nx, int64_t ny, int64_t nz, double dx, double dy, double dz,
                         const double* verts, int mode) {
  using namespace cfdb_geom;
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
  const Lattice L{nx, ny, nz, dx, dy, dz, verts};

#pragma omp parallel for schedule(static)
  for (int64_t x = 0; x < nx; ++x)
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t z = 0; z < nz; ++z) {
        const P3 c = L.center(x, y, z);
        const int64_t i = L.id(x, y, z);
        g.center[i] = c.x; g.center[n + i] = c.y; g.center[2 * n + i] = c.z;
      }
  auto center_of = [&](int64_t x, int64_t y, int64_t z) {
    const int64_t j = L.id(x, y, z);
    return P3{g.center[j], g.center[n + j], g.center[2 * n + j]};
  };

#pragma omp parallel for schedule(static)
  for (int64_t x = 0; x < nx; ++x)
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t z = 0; z < nz; ++z) {
        const int64_t i = L.id(x, y, z);
        bool bnd = false;
        auto store = [&](int f, const CellFace& o) {
          const int64_t k6 = int64_t(f) * n + i;
          g.normal[k6] = o.uns.x; g.normal[6 * n + k6] = o.uns.y; g.normal[12 * n + k6] = o.uns.z;
          g.normal_alt[k6] = o.good.x; g.normal_alt[6 * n + k6] = o.good.y; g.normal_alt[12 * n + k6] = o.good.z;
          g.area[k6] = o.area;
          g.alpha[k6] = o.alpha;
          g.len[k6] = o.len;
          g.ids[k6] = o.id;
          g.ibf[k6] = o.ibf;
        };
        const double vol = cell_geometry(L, x, y, z, mode, center_of, store, &bnd);
        g.volume[i] = vol;
        g.isb[i] = bnd ? 1.0 : 0.0;
      }
  return true;
}
