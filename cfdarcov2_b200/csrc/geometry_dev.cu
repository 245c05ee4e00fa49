// Device builder of the per-face geometry arrays the plain kernels read
// (normal, normal_alt, area, alpha, len, volume, is_boundary and the int32
// neighbour ids): one thread per cell evaluates geometry_cell.hpp's formulas
// in double, each operation separately rounded (this file is compiled with
// --fmad=false), so the arrays hold the host builder's doubles, converted to
// the storage type.  A 400^3 lattice takes milliseconds here instead of the
// host pass over 64M cells plus the upload of ~16 GB.
#include "cfdb_internal.hpp"
#include "geometry_cell.hpp"

CFDB_MODULE_ANCHOR

namespace {

using cfdb_geom::CellFace;
using cfdb_geom::Lattice;
using cfdb_geom::P3;

template <class T>
__global__ void __launch_bounds__(128) plain_geometry_k(Lattice L, int mode, T* __restrict__ normal,
                                                        T* __restrict__ normal_alt, T* __restrict__ area,
                                                        T* __restrict__ alpha, T* __restrict__ len,
                                                        T* __restrict__ volume, T* __restrict__ isb,
                                                        int32_t* __restrict__ ids) {
  const int64_t n = L.nx * L.ny * L.nz, plane = L.ny * L.nz;
  auto center_of = [&](int64_t x, int64_t y, int64_t z) { return L.center(x, y, z); };
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t x = i / plane, r = i - x * plane, y = r / L.nz, z = r - y * L.nz;
    bool bnd = false;
    auto store = [&](int f, const CellFace& o) {
      const int64_t k6 = int64_t(f) * n + i;
      normal[k6] = T(o.uns.x);
      normal[6 * n + k6] = T(o.uns.y);
      normal[12 * n + k6] = T(o.uns.z);
      normal_alt[k6] = T(o.good.x);
      normal_alt[6 * n + k6] = T(o.good.y);
      normal_alt[12 * n + k6] = T(o.good.z);
      area[k6] = T(o.area);
      alpha[k6] = T(o.alpha);
      len[k6] = T(o.len);
      if (ids) ids[k6] = int32_t(o.id);
    };
    const double vol = cfdb_geom::cell_geometry(L, x, y, z, mode, center_of, store, &bnd);
    volume[i] = T(vol);
    isb[i] = T(bnd ? 1.0 : 0.0);
  }
}

}  // namespace

// Allocates and fills p (and m->d_ids when it is not built yet) on the
// context's stream; synchronises before returning.
int cfdb_build_plain_device(cfdb_mesh* m, int dtype, PlainGeomDev& p) {
  cfdb_ctx* ctx = m->ctx;
  const int64_t n = m->n;
  if (6 * n > int64_t(INT32_MAX)) return cfdb_fail(ctx, CFDB_EUNSUPPORTED, "mesh too large for int32 face ids");
  const int64_t es = dtype == CFDB_F64 ? 8 : 4;
  void** arrays[] = {&p.normal, &p.normal_alt, &p.area, &p.alpha, &p.len, &p.volume, &p.isb};
  const int64_t counts[] = {18 * n, 18 * n, 6 * n, 6 * n, 6 * n, n, n};
  for (int k = 0; k < 7; ++k)
    if (int rc = cfdb_dev_alloc(ctx, counts[k] * es, arrays[k])) return rc;
  const bool need_ids = m->d_ids == nullptr;
  if (need_ids)
    if (int rc = cfdb_dev_alloc(ctx, int64_t(sizeof(int32_t)) * 6 * n, reinterpret_cast<void**>(&m->d_ids))) return rc;
  double* dverts = nullptr;
  if (!m->uniform) {
    const int64_t bytes = int64_t(sizeof(double)) * int64_t(m->verts.size());
    if (int rc = cfdb_dev_alloc(ctx, bytes, reinterpret_cast<void**>(&dverts))) return rc;
    CFDB_CUDA(ctx, cudaMemcpyAsync(dverts, m->verts.data(), size_t(bytes), cudaMemcpyHostToDevice, ctx->stream));
  }
  const Lattice L{m->nx, m->ny, m->nz, m->dx, m->dy, m->dz, dverts};
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  const int64_t want = (n + 127) / 128;
  const unsigned blocks = unsigned(want < int64_t(sms) * 16 ? (want > 0 ? want : 1) : int64_t(sms) * 16);
  int32_t* ids = need_ids ? m->d_ids : nullptr;
  if (dtype == CFDB_F64)
    plain_geometry_k<double><<<blocks, 128, 0, ctx->stream>>>(
        L, m->geom_mode, static_cast<double*>(p.normal), static_cast<double*>(p.normal_alt),
        static_cast<double*>(p.area), static_cast<double*>(p.alpha), static_cast<double*>(p.len),
        static_cast<double*>(p.volume), static_cast<double*>(p.isb), ids);
  else
    plain_geometry_k<float><<<blocks, 128, 0, ctx->stream>>>(
        L, m->geom_mode, static_cast<float*>(p.normal), static_cast<float*>(p.normal_alt),
        static_cast<float*>(p.area), static_cast<float*>(p.alpha), static_cast<float*>(p.len),
        static_cast<float*>(p.volume), static_cast<float*>(p.isb), ids);
  CFDB_CUDA(ctx, cudaGetLastError());
  CFDB_LAUNCHED(ctx);
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  cfdb_dev_free(ctx, dverts);
  return CFDB_OK;
}

// ---- exact lattices --------------------------------------------------------
namespace {

struct FaceSample {
  float normal[18], normal_alt[18], area[6], alpha[6], len[6], volume;
};

__device__ __forceinline__ void sample_cell(const Lattice& L, int64_t x, int64_t y, int64_t z, int mode,
                                            FaceSample* s) {
  auto center_of = [&](int64_t a, int64_t b, int64_t c) { return L.center(a, b, c); };
  bool bnd = false;
  auto store = [&](int f, const CellFace& o) {
    s->normal[f] = float(o.uns.x);
    s->normal[6 + f] = float(o.uns.y);
    s->normal[12 + f] = float(o.uns.z);
    s->normal_alt[f] = float(o.good.x);
    s->normal_alt[6 + f] = float(o.good.y);
    s->normal_alt[12 + f] = float(o.good.z);
    s->area[f] = float(o.area);
    s->alpha[f] = float(o.alpha);
    s->len[f] = float(o.len);
  };
  s->volume = float(cfdb_geom::cell_geometry(L, x, y, z, mode, center_of, store, &bnd));
}

// the first and the last cell: between them every slot is seen once as a
// wall face and (where the dimension has two cells or more) once inside
__global__ void lattice_sample_k(Lattice L, int mode, FaceSample* out) {
  if (threadIdx.x == 0) sample_cell(L, 0, 0, 0, mode, &out[0]);
  if (threadIdx.x == 1) sample_cell(L, L.nx - 1, L.ny - 1, L.nz - 1, mode, &out[1]);
}

__device__ __forceinline__ bool same(float a, float b) { return __float_as_uint(a) == __float_as_uint(b); }

// bad |= 1 when a cell's FP32 face values or neighbour ids differ from the constants
__global__ void __launch_bounds__(128) lattice_check_k(Lattice L, int mode, cfdb_lattice_geometry c, int* bad) {
  const int64_t n = L.nx * L.ny * L.nz, plane = L.ny * L.nz;
  auto center_of = [&](int64_t a, int64_t b, int64_t cz) { return L.center(a, b, cz); };
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t x = i / plane, r = i - x * plane, y = r / L.nz, z = r - y * L.nz;
    bool bnd = false;
    bool ok = true;
    auto check = [&](int f, const CellFace& o) {
      const bool wall = f == 0 ? z == 0 : f == 1 ? z == L.nz - 1 : f == 2 ? y == 0 : f == 3 ? y == L.ny - 1
                      : f == 4 ? x == 0 : x == L.nx - 1;
      const int64_t step = f == 0 ? -1 : f == 1 ? 1 : f == 2 ? -L.nz : f == 3 ? L.nz : f == 4 ? -plane : plane;
      const int w = wall ? 1 : 0;
      ok = ok && same(float(o.uns.x), c.normal[f]) && same(float(o.uns.y), c.normal[6 + f]) &&
           same(float(o.uns.z), c.normal[12 + f]) && same(float(o.good.x), c.normal_alt[f]) &&
           same(float(o.good.y), c.normal_alt[6 + f]) && same(float(o.good.z), c.normal_alt[12 + f]) &&
           same(float(o.area), c.area[f]) && same(float(o.alpha), c.alpha[w * 6 + f]) &&
           same(float(o.len), c.len[w * 6 + f]) && o.id == (w ? i : i + step);
    };
    const double vol = cfdb_geom::cell_geometry(L, x, y, z, mode, center_of, check, &bnd);
    ok = ok && same(float(vol), c.volume);
    if (!ok) atomicOr(bad, 1);
  }
}

}  // namespace

// Fills out with the lattice constants and exact = 1 when every cell's FP32
// face values equal them; exact = 0 otherwise.  Synchronises the stream.
int cfdb_check_lattice_device(cfdb_mesh* m, cfdb_lattice_geometry* out) {
  cfdb_ctx* ctx = m->ctx;
  *out = cfdb_lattice_geometry{};
  out->nx = m->nx;
  out->ny = m->ny;
  out->nz = m->nz;
  if (!m->uniform || m->n == 0) return CFDB_OK;
  const Lattice L{m->nx, m->ny, m->nz, m->dx, m->dy, m->dz, nullptr};
  FaceSample* d = nullptr;
  if (int rc = cfdb_dev_alloc(ctx, int64_t(2 * sizeof(FaceSample) + sizeof(int)), reinterpret_cast<void**>(&d)))
    return rc;
  int* bad = reinterpret_cast<int*>(d + 2);
  CFDB_CUDA(ctx, cudaMemsetAsync(bad, 0, sizeof(int), ctx->stream));
  lattice_sample_k<<<1, 32, 0, ctx->stream>>>(L, m->geom_mode, d);
  CFDB_CUDA(ctx, cudaGetLastError());
  CFDB_LAUNCHED(ctx);
  FaceSample s[2];
  CFDB_CUDA(ctx, cudaMemcpyAsync(s, d, sizeof(s), cudaMemcpyDeviceToHost, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  // slots 0, 2, 4 (the - faces) are walls of the first cell, 1, 3, 5 of the last
  const int64_t dims[3] = {m->nz, m->ny, m->nx};  // slot pair 0/1: z, 2/3: y, 4/5: x
  for (int f = 0; f < 6; ++f) {
    const FaceSample& w = s[f % 2 == 0 ? 0 : 1];
    const FaceSample& in = dims[f / 2] > 1 ? s[f % 2 == 0 ? 1 : 0] : w;
    for (int dd = 0; dd < 3; ++dd) {
      out->normal[dd * 6 + f] = w.normal[dd * 6 + f];
      out->normal_alt[dd * 6 + f] = w.normal_alt[dd * 6 + f];
    }
    out->area[f] = w.area[f];
    out->alpha[6 + f] = w.alpha[f];
    out->len[6 + f] = w.len[f];
    out->alpha[f] = in.alpha[f];
    out->len[f] = in.len[f];
  }
  out->volume = s[0].volume;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  const int64_t want = (m->n + 127) / 128;
  const unsigned blocks = unsigned(want < int64_t(sms) * 16 ? want : int64_t(sms) * 16);
  lattice_check_k<<<blocks, 128, 0, ctx->stream>>>(L, m->geom_mode, *out, bad);
  CFDB_CUDA(ctx, cudaGetLastError());
  CFDB_LAUNCHED(ctx);
  int h_bad = 1;
  CFDB_CUDA(ctx, cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  cfdb_dev_free(ctx, d);
  out->exact = h_bad ? 0 : 1;
  return CFDB_OK;
}
