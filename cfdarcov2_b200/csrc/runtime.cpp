// Host runtime of libcfdb: contexts, errors, device memory, meshes and their
// geometry uploads.  Replaces CFDArcoGlobalInit (src/cfdarcho_main_3d.cpp),
// CudaDataMatrix + the RMM pool (include/cuda_data_matrix.hpp,
// include/pool_allocator.hpp) and CudaMesh3D::host_to_device
// (include/mesh3d.hpp:209-236) with library-owned buffers, status codes and
// no per-step allocation.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include <cuda.h>

#include "cfdb_internal.hpp"

namespace {
thread_local std::string g_err_noctx;

std::string vformat(const char* fmt, va_list ap) {
  char buf[1024];
  vsnprintf(buf, sizeof(buf), fmt, ap);
  return std::string(buf);
}
}  // namespace

int cfdb_fail(cfdb_ctx* ctx, int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::string s = vformat(fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = s; else g_err_noctx = s;
  return code;
}

int cfdb_cuda_fail(cfdb_ctx* ctx, cudaError_t e, const char* what) {
  cudaGetLastError();  // clear a sticky-free error so the next call starts clean
  return cfdb_fail(ctx, e == cudaErrorMemoryAllocation ? CFDB_ENOMEM : CFDB_ECUDA, "%s: %s (%s)", what,
                   cudaGetErrorString(e), cudaGetErrorName(e));
}

int cfdb_dev_alloc(cfdb_ctx* ctx, int64_t bytes, void** out) {
  *out = nullptr;
  if (bytes <= 0) bytes = 16;
  if (ctx->budget > 0 && ctx->allocated + bytes > ctx->budget)
    return cfdb_fail(ctx, CFDB_ENOMEM, "allocation of %lld bytes exceeds the context budget (%lld of %lld used)",
                     (long long)bytes, (long long)ctx->allocated, (long long)ctx->budget);
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, size_t(bytes));
  if (e != cudaSuccess) return cfdb_cuda_fail(ctx, e, "cudaMalloc");
  ctx->allocs[p] = bytes;
  ctx->allocated += bytes;
  *out = p;
  return CFDB_OK;
}

void cfdb_dev_free(cfdb_ctx* ctx, void* p) {
  if (!p || !ctx) return;
  auto it = ctx->allocs.find(p);
  if (it != ctx->allocs.end()) {
    ctx->allocated -= it->second;
    ctx->allocs.erase(it);
  }
  cudaFree(p);
}

// ---- module loading -----------------------------------------------------------
namespace {
std::vector<const void*>& module_anchors() {
  static std::vector<const void*> v;
  return v;
}

template <class F> F driver_fn(const char* name) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
    return nullptr;
  return reinterpret_cast<F>(p);
}

// Loads every kernel of the registered modules on the current device, once
// per device and process.  Best effort: a driver without the enumeration
// calls (before CUDA 12.4) leaves loading to the first launches.
void load_modules(int device) {
  static std::mutex mu;
  static bool done[kMaxDevices] = {};
  std::lock_guard<std::mutex> lock(mu);
  if (device < 0 || device >= kMaxDevices || done[device]) return;
  done[device] = true;
  using GetModule = CUresult (*)(CUmodule*, CUfunction);
  using Count = CUresult (*)(unsigned int*, CUmodule);
  using Enumerate = CUresult (*)(CUfunction*, unsigned int, CUmodule);
  using Load = CUresult (*)(CUfunction);
  auto get_module = driver_fn<GetModule>("cuFuncGetModule");
  auto count = driver_fn<Count>("cuModuleGetFunctionCount");
  auto enumerate = driver_fn<Enumerate>("cuModuleEnumerateFunctions");
  auto load = driver_fn<Load>("cuFuncLoad");
  if (!get_module || !count || !enumerate || !load) return;
  for (const void* anchor : module_anchors()) {
    cudaFunction_t f = nullptr;
    if (cudaGetFuncBySymbol(&f, anchor) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    CUmodule mod = nullptr;
    unsigned int n = 0;
    if (get_module(&mod, reinterpret_cast<CUfunction>(f)) != CUDA_SUCCESS || count(&n, mod) != CUDA_SUCCESS || n == 0)
      continue;
    std::vector<CUfunction> fns(n);
    if (enumerate(fns.data(), n, mod) != CUDA_SUCCESS) continue;
    for (CUfunction fn : fns) load(fn);
  }
}

// The context's stream-ordered pool, created with the context and grown by
// one small block so that the first workspace of a step does not create it.
int make_pool(cfdb_ctx* ctx) {
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = ctx->device;
  CFDB_CUDA(ctx, cudaMemPoolCreate(&ctx->pool, &props));
  uint64_t keep = UINT64_MAX;  // never hand freed blocks back on synchronisation
  CFDB_CUDA(ctx, cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep));
  void* p = nullptr;
  CFDB_CUDA(ctx, cudaMallocFromPoolAsync(&p, 1 << 20, ctx->pool, ctx->stream));
  CFDB_CUDA(ctx, cudaFreeAsync(p, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CFDB_OK;
}
}  // namespace

int cfdb_register_module(const void* anchor_kernel) {
  module_anchors().push_back(anchor_kernel);
  return 0;
}

int cfdb_ws_alloc(cfdb_ctx* ctx, int64_t bytes, void** out) {
  *out = nullptr;
  if (bytes <= 0) bytes = 16;
  if (ctx->budget > 0 && ctx->allocated + bytes > ctx->budget)
    return cfdb_fail(ctx, CFDB_ENOMEM, "workspace of %lld bytes exceeds the context budget (%lld of %lld used)",
                     (long long)bytes, (long long)ctx->allocated, (long long)ctx->budget);
  if (!ctx->pool)
    if (int rc = make_pool(ctx)) return rc;
  void* p = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&p, size_t(bytes), ctx->pool, ctx->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    // blocks cached for other sizes may be what is missing: return them and retry once
    cudaStreamSynchronize(ctx->stream);
    cudaMemPoolTrimTo(ctx->pool, 0);
    e = cudaMallocFromPoolAsync(&p, size_t(bytes), ctx->pool, ctx->stream);
    if (e != cudaSuccess) return cfdb_cuda_fail(ctx, e, "cudaMallocFromPoolAsync");
  }
  ctx->ws[p] = bytes;
  ctx->allocated += bytes;
  *out = p;
  return CFDB_OK;
}

void cfdb_ws_free(cfdb_ctx* ctx, void* p) {
  if (!p || !ctx) return;
  auto it = ctx->ws.find(p);
  if (it == ctx->ws.end()) return;
  ctx->allocated -= it->second;
  ctx->ws.erase(it);
  cudaFreeAsync(p, ctx->stream);
}

extern "C" int cfdb_ctx_launch_count(const cfdb_ctx* ctx, int64_t* out) {
  if (!ctx || !out) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_ctx_launch_count: bad arguments");
  *out = ctx->launches;
  return CFDB_OK;
}


extern "C" int cfdb_ctx_set_wait_limit(cfdb_ctx* ctx, int64_t cycles, int32_t missing_plane) {
  if (!ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_ctx_set_wait_limit: ctx is NULL");
  if (cycles < 1000) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_ctx_set_wait_limit: cycles must be >= 1000");
  if (missing_plane < -1) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_ctx_set_wait_limit: missing_plane must be >= -1");
  ctx->wait_cycles = cycles;
  ctx->missing_plane = missing_plane;
  cfdb_graphs_clear(ctx);  // recorded launches carry the old values
  return CFDB_OK;
}

extern "C" int cfdb_ctx_trim(cfdb_ctx* ctx) {
  if (!ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_ctx_trim: ctx is NULL");
  if (!ctx->pool) return CFDB_OK;
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  CFDB_CUDA(ctx, cudaMemPoolTrimTo(ctx->pool, 0));
  return CFDB_OK;
}

extern "C" int cfdb_abi_version(void) { return CFDB_ABI_VERSION; }

extern "C" int cfdb_ctx_create(int device, cfdb_ctx** out) {
  if (!out) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_ctx_create: out is NULL");
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess) return cfdb_cuda_fail(nullptr, e, "cudaGetDeviceCount");
  if (device < 0 || device >= count)
    return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_ctx_create: device %d out of range (%d devices)", device, count);
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return cfdb_cuda_fail(nullptr, e, "cudaSetDevice");
  auto* ctx = new (std::nothrow) cfdb_ctx();
  if (!ctx) return cfdb_fail(nullptr, CFDB_ENOMEM, "cfdb_ctx_create: host allocation failed");
  ctx->device = device;
  cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  int rc = cfdb_dev_alloc(ctx, sizeof(int) * 4, reinterpret_cast<void**>(&ctx->d_error));
  if (rc) {
    g_err_noctx = ctx->err;
    delete ctx;
    return rc;
  }
  e = cudaMemset(ctx->d_error, 0, sizeof(int) * 4);
  if (e != cudaSuccess) {
    int r = cfdb_cuda_fail(nullptr, e, "cudaMemset");
    cfdb_dev_free(ctx, ctx->d_error);
    delete ctx;
    return r;
  }
  if ((rc = make_pool(ctx))) {
    g_err_noctx = ctx->err;
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    cfdb_dev_free(ctx, ctx->d_error);
    delete ctx;
    return rc;
  }
  load_modules(device);
  *out = ctx;
  return CFDB_OK;
}

extern "C" int cfdb_ctx_destroy(cfdb_ctx* ctx) {
  if (!ctx) return CFDB_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cfdb_graphs_clear(ctx);
  cfdb_jit_release(ctx);
  if (ctx->capture_stream) cudaStreamDestroy(ctx->capture_stream);
  auto children = std::move(ctx->children);
  for (auto& kv : children) kv.second();
  for (auto& kv : ctx->allocs) cudaFree(kv.first);
  ctx->allocs.clear();
  if (ctx->pool) {
    for (auto& kv : ctx->ws) cudaFreeAsync(kv.first, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    cudaMemPoolDestroy(ctx->pool);
  }
  delete ctx;
  return CFDB_OK;
}

extern "C" const char* cfdb_last_error(const cfdb_ctx* ctx) {
  return ctx ? ctx->err.c_str() : g_err_noctx.c_str();
}

extern "C" int cfdb_ctx_set_stream(cfdb_ctx* ctx, void* stream) {
  if (!ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_ctx_set_stream: ctx is NULL");
  ctx->stream = static_cast<cudaStream_t>(stream);
  return CFDB_OK;
}

int cfdb_check_device_error(cfdb_ctx* ctx) {
  int err = 0;
  CFDB_CUDA(ctx, cudaMemcpyAsync(&err, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (!err) return CFDB_OK;
  CFDB_CUDA(ctx, cudaMemsetAsync(ctx->d_error, 0, sizeof(int), ctx->stream));
  switch (err) {
    case 1: return cfdb_fail(ctx, CFDB_ETIMEOUT, "a bounded device wait gave up (a staged copy or a neighbouring cluster's plane never arrived)");
    case 2: return cfdb_fail(ctx, CFDB_ECUDA, "a sweep kernel found its shared memory misaligned for TMA");
    case 3: return cfdb_fail(ctx, CFDB_ECUDA, "a sweep kernel was launched with less shared memory than its layout");
    default: return cfdb_fail(ctx, CFDB_ECUDA, "device error word %d", err);
  }
}

extern "C" int cfdb_sync(cfdb_ctx* ctx) {
  if (!ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_sync: ctx is NULL");
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return cfdb_check_device_error(ctx);
}

extern "C" int cfdb_ctx_set_alloc_budget(cfdb_ctx* ctx, int64_t bytes) {
  if (!ctx || bytes < 0) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_ctx_set_alloc_budget: bad arguments");
  ctx->budget = bytes;
  return CFDB_OK;
}

extern "C" int cfdb_ctx_allocated_bytes(const cfdb_ctx* ctx, int64_t* out) {
  if (!ctx || !out) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_ctx_allocated_bytes: bad arguments");
  *out = ctx->allocated;
  return CFDB_OK;
}

extern "C" int cfdb_alloc(cfdb_ctx* ctx, int64_t bytes, void** out) {
  if (!ctx || !out || bytes < 0) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_alloc: bad arguments");
  return cfdb_dev_alloc(ctx, bytes, out);
}

extern "C" int cfdb_free(cfdb_ctx* ctx, void* ptr) {
  if (!ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_free: ctx is NULL");
  if (ptr && !ctx->allocs.count(ptr)) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_free: pointer not owned by ctx");
  cudaStreamSynchronize(ctx->stream);
  cfdb_dev_free(ctx, ptr);
  return CFDB_OK;
}

extern "C" int cfdb_upload(cfdb_ctx* ctx, void* dst, const void* src, int64_t bytes) {
  if (!ctx || !dst || !src || bytes < 0) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_upload: bad arguments");
  CFDB_CUDA(ctx, cudaMemcpyAsync(dst, src, size_t(bytes), cudaMemcpyHostToDevice, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CFDB_OK;
}

extern "C" int cfdb_download(cfdb_ctx* ctx, void* dst, const void* src, int64_t bytes) {
  if (!ctx || !dst || !src || bytes < 0) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_download: bad arguments");
  CFDB_CUDA(ctx, cudaMemcpyAsync(dst, src, size_t(bytes), cudaMemcpyDeviceToHost, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CFDB_OK;
}

extern "C" int cfdb_upload_async(cfdb_ctx* ctx, void* dst, const void* src, int64_t bytes) {
  if (!ctx || !dst || !src || bytes < 0) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_upload_async: bad arguments");
  CFDB_CUDA(ctx, cudaMemcpyAsync(dst, src, size_t(bytes), cudaMemcpyHostToDevice, ctx->stream));
  return CFDB_OK;
}

extern "C" int cfdb_download_async(cfdb_ctx* ctx, void* dst, const void* src, int64_t bytes) {
  if (!ctx || !dst || !src || bytes < 0) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_download_async: bad arguments");
  CFDB_CUDA(ctx, cudaMemcpyAsync(dst, src, size_t(bytes), cudaMemcpyDeviceToHost, ctx->stream));
  return CFDB_OK;
}

// ---------------------------------------------------------------------------
// meshes
// ---------------------------------------------------------------------------
namespace {
int check_dims(cfdb_ctx* ctx, int64_t nx, int64_t ny, int64_t nz, double dx, double dy, double dz) {
  if (nx < 1 || ny < 1 || nz < 1)
    return cfdb_fail(ctx, CFDB_EINVAL, "mesh dimensions must be >= 1 (got %lld x %lld x %lld)", (long long)nx,
                     (long long)ny, (long long)nz);
  if (!(dx > 0) || !(dy > 0) || !(dz > 0) || !std::isfinite(dx) || !std::isfinite(dy) || !std::isfinite(dz))
    return cfdb_fail(ctx, CFDB_EINVAL, "mesh spacings must be finite and > 0");
  const double cells = double(nx) * double(ny) * double(nz);
  if (cells > double(INT32_MAX))
    return cfdb_fail(ctx, CFDB_EINVAL, "mesh of %.0f cells exceeds the 2^31-1 cell limit of int32 indexing", cells);
  return CFDB_OK;
}
}  // namespace

static uint64_t next_mesh_uid() {
  static std::atomic<uint64_t> uid{0};
  return ++uid;
}

extern "C" int cfdb_mesh_create_structured(cfdb_ctx* ctx, int64_t nx, int64_t ny, int64_t nz, double dx,
                                           double dy, double dz, cfdb_mesh** out) {
  if (!out) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_mesh_create_structured: out is NULL");
  *out = nullptr;
  if (int rc = check_dims(ctx, nx, ny, nz, dx, dy, dz)) return rc;
  auto* m = new (std::nothrow) cfdb_mesh();
  if (!m) return cfdb_fail(ctx, CFDB_ENOMEM, "host allocation failed");
  m->ctx = ctx;
  m->uid = next_mesh_uid();
  m->nx = nx; m->ny = ny; m->nz = nz; m->n = nx * ny * nz;
  m->dx = dx; m->dy = dy; m->dz = dz;
  m->uniform = true;
  cfdb_adopt(ctx, m, [m] { cfdb_mesh_orphan(m); });
  *out = m;
  return CFDB_OK;
}

extern "C" int cfdb_mesh_create_from_vertices(cfdb_ctx* ctx, int64_t nx, int64_t ny, int64_t nz, double dx,
                                              double dy, double dz, const double* vertices, int flags,
                                              cfdb_mesh** out) {
  if (!out || !vertices) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_mesh_create_from_vertices: NULL argument");
  *out = nullptr;
  if (int rc = check_dims(ctx, nx, ny, nz, dx, dy, dz)) return rc;
  if (flags & ~CFDB_MESH_COMPAT_AREA) return cfdb_fail(ctx, CFDB_EINVAL, "unknown mesh flags 0x%x", flags);
  const int64_t nv = (nx + 1) * (ny + 1) * (nz + 1);
  for (int64_t k = 0; k < 3 * nv; ++k)
    if (!std::isfinite(vertices[k])) return cfdb_fail(ctx, CFDB_EINVAL, "vertex coordinate %lld is not finite", (long long)k);
  auto* m = new (std::nothrow) cfdb_mesh();
  if (!m) return cfdb_fail(ctx, CFDB_ENOMEM, "host allocation failed");
  m->ctx = ctx;
  m->uid = next_mesh_uid();
  m->nx = nx; m->ny = ny; m->nz = nz; m->n = nx * ny * nz;
  m->dx = dx; m->dy = dy; m->dz = dz;
  m->uniform = false;
  m->geom_mode = (flags & CFDB_MESH_COMPAT_AREA) ? 1 : 2;
  try {
    m->verts.assign(vertices, vertices + 3 * nv);
  } catch (const std::bad_alloc&) {
    delete m;
    return cfdb_fail(ctx, CFDB_ENOMEM, "host allocation failed");
  }
  if (int rc = cfdb_mesh_need_host_geom(m)) {
    delete m;
    return rc;
  }
  // Reject tangled cells.  The outward normal comes from a sign test against
  // the cell centre (src/mesh3d.cpp:84-88), so the volume stays positive even
  // when a face has folded over; instead every face's outward normal must lie
  // on its topological side: along the unsigned normal for the +x/+y/+z slots
  // (1, 3, 5), against it for the -slots (0, 2, 4).
  {
    const HostGeom& g = *m->geom;
    const int64_t n = m->n;
    for (int64_t i = 0; i < n; ++i) {
      bool ok = g.volume[i] > 0;
      for (int f = 0; f < 6 && ok; ++f) {
        const int64_t k6 = int64_t(f) * n + i;
        const double d = g.normal_alt[k6] * g.normal[k6] + g.normal_alt[6 * n + k6] * g.normal[6 * n + k6] +
                         g.normal_alt[12 * n + k6] * g.normal[12 * n + k6];
        ok = (f & 1) ? d > 0 : d < 0;
      }
      if (!ok) {
        delete m;
        return cfdb_fail(ctx, CFDB_EINVAL, "cell %lld is tangled (a face normal or the volume is inverted)",
                         (long long)i);
      }
    }
  }
  cfdb_adopt(ctx, m, [m] { cfdb_mesh_orphan(m); });
  *out = m;
  return CFDB_OK;
}

static void free_plain(cfdb_ctx* ctx, PlainGeomDev& p) {
  void** ptrs[] = {&p.normal, &p.normal_alt, &p.area, &p.alpha, &p.len, &p.volume, &p.isb, &p.stab_tmp};
  for (void** q : ptrs) {
    cfdb_dev_free(ctx, *q);
    *q = nullptr;
  }
  p.ready = false;
}

// The context is going away: its allocations are freed with it.
void cfdb_mesh_orphan(cfdb_mesh* m) {
  m->ctx = nullptr;
  m->plain[0] = PlainGeomDev();
  m->plain[1] = PlainGeomDev();
  m->d_ids = nullptr;
  m->compact = CompactGeomDev();
}

extern "C" int cfdb_mesh_destroy(cfdb_mesh* m) {
  if (!m) return CFDB_OK;
  if (m->ctx) {
    cfdb_release(m->ctx, m);
    cudaStreamSynchronize(m->ctx->stream);
    free_plain(m->ctx, m->plain[0]);
    free_plain(m->ctx, m->plain[1]);
    cfdb_dev_free(m->ctx, m->d_ids);
    cfdb_dev_free(m->ctx, m->compact.S);
  }
  delete m;
  return CFDB_OK;
}

extern "C" int cfdb_mesh_info(const cfdb_mesh* m, int64_t dims[3], double spacing[3], int* is_uniform) {
  if (!m) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_mesh_info: mesh is NULL");
  if (dims) { dims[0] = m->nx; dims[1] = m->ny; dims[2] = m->nz; }
  if (spacing) { spacing[0] = m->dx; spacing[1] = m->dy; spacing[2] = m->dz; }
  if (is_uniform) *is_uniform = m->uniform ? 1 : 0;
  return CFDB_OK;
}

int cfdb_mesh_need_host_geom(cfdb_mesh* m) {
  if (m->geom) return CFDB_OK;
  auto g = std::unique_ptr<HostGeom>(new (std::nothrow) HostGeom());
  if (!g) return cfdb_fail(m->ctx, CFDB_ENOMEM, "host allocation failed");
  if (!cfdb_build_geometry(*g, m->nx, m->ny, m->nz, m->dx, m->dy, m->dz, m->uniform ? nullptr : m->verts.data(),
                           m->geom_mode))
    return cfdb_fail(m->ctx, CFDB_ENOMEM, "host geometry of %lld cells does not fit in host memory", (long long)m->n);
  m->geom = std::move(g);
  return CFDB_OK;
}

extern "C" int cfdb_mesh_geometry(const cfdb_mesh* cm, int which, double* out) {
  cfdb_mesh* m = const_cast<cfdb_mesh*>(cm);
  if (!m || !out) return cfdb_fail(m ? m->ctx : nullptr, CFDB_EINVAL, "cfdb_mesh_geometry: NULL argument");
  if (int rc = cfdb_mesh_need_host_geom(m)) return rc;
  const HostGeom& g = *m->geom;
  const std::vector<double>* src = nullptr;
  switch (which) {
    case CFDB_GEOM_NORMAL: src = &g.normal; break;
    case CFDB_GEOM_NORMAL_ALT: src = &g.normal_alt; break;
    case CFDB_GEOM_AREA: src = &g.area; break;
    case CFDB_GEOM_ALPHA_D: src = &g.alpha; break;
    case CFDB_GEOM_LEN_C2F: src = &g.len; break;
    case CFDB_GEOM_VOLUME: src = &g.volume; break;
    case CFDB_GEOM_CENTER: src = &g.center; break;
    case CFDB_GEOM_IS_BOUNDARY: src = &g.isb; break;
    default: return cfdb_fail(m->ctx, CFDB_EINVAL, "cfdb_mesh_geometry: unknown array %d", which);
  }
  std::memcpy(out, src->data(), sizeof(double) * src->size());
  return CFDB_OK;
}

extern "C" int cfdb_mesh_ids(const cfdb_mesh* cm, int64_t* ids, int64_t* ibf) {
  cfdb_mesh* m = const_cast<cfdb_mesh*>(cm);
  if (!m) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_mesh_ids: mesh is NULL");
  if (int rc = cfdb_mesh_need_host_geom(m)) return rc;
  if (ids) std::memcpy(ids, m->geom->ids.data(), sizeof(int64_t) * 6 * m->n);
  if (ibf) std::memcpy(ibf, m->geom->ibf.data(), sizeof(int64_t) * 6 * m->n);
  return CFDB_OK;
}

int cfdb_check_mesh(cfdb_ctx* ctx, cfdb_mesh* m) {
  if (!ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "ctx is NULL");
  if (!m) return cfdb_fail(ctx, CFDB_EINVAL, "mesh is NULL");
  if (m->ctx != ctx) return cfdb_fail(ctx, CFDB_EINVAL, "mesh belongs to another context (or is host-only)");
  return CFDB_OK;
}

namespace {
template <class T>
int upload_as(cfdb_ctx* ctx, const double* src, int64_t count, void** dst) {
  std::vector<T> tmp;
  try {
    tmp.resize(size_t(count));
  } catch (const std::bad_alloc&) {
    return cfdb_fail(ctx, CFDB_ENOMEM, "host staging allocation failed");
  }
  for (int64_t k = 0; k < count; ++k) tmp[k] = T(src[k]);
  if (int rc = cfdb_dev_alloc(ctx, int64_t(sizeof(T)) * count, dst)) return rc;
  CFDB_CUDA(ctx, cudaMemcpy(*dst, tmp.data(), sizeof(T) * size_t(count), cudaMemcpyHostToDevice));
  return CFDB_OK;
}
}  // namespace

int cfdb_mesh_need_plain(cfdb_mesh* m, int dtype) {
  PlainGeomDev& p = m->plain[dtype == CFDB_F64 ? 1 : 0];
  if (p.ready) return CFDB_OK;
  CFDB_CUDA(m->ctx, cudaSetDevice(m->ctx->device));
  if (int rc = cfdb_build_plain_device(m, dtype, p)) {
    free_plain(m->ctx, p);
    return rc;
  }
  p.ready = true;
  return CFDB_OK;
}

extern "C" int cfdb_mesh_plain_geometry(cfdb_mesh* m, cfdb_plain_geometry* out) {
  if (!out) return cfdb_fail(m ? m->ctx : nullptr, CFDB_EINVAL, "cfdb_mesh_plain_geometry: out is NULL");
  if (!m || !m->ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_mesh_plain_geometry: mesh is NULL or host-only");
  CFDB_CUDA(m->ctx, cudaSetDevice(m->ctx->device));
  if (int rc = cfdb_mesh_need_plain(m, CFDB_F32)) return rc;
  const PlainGeomDev& p = m->plain[0];
  out->ids = m->d_ids;
  out->normal = static_cast<const float*>(p.normal);
  out->normal_alt = static_cast<const float*>(p.normal_alt);
  out->area = static_cast<const float*>(p.area);
  out->alpha = static_cast<const float*>(p.alpha);
  out->len = static_cast<const float*>(p.len);
  out->volume = static_cast<const float*>(p.volume);
  out->n = m->n;
  return CFDB_OK;
}

extern "C" int cfdb_mesh_lattice_geometry(cfdb_mesh* m, cfdb_lattice_geometry* out) {
  if (!out) return cfdb_fail(m ? m->ctx : nullptr, CFDB_EINVAL, "cfdb_mesh_lattice_geometry: out is NULL");
  if (!m || !m->ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_mesh_lattice_geometry: mesh is NULL or host-only");
  if (m->lattice_state == 0) {
    CFDB_CUDA(m->ctx, cudaSetDevice(m->ctx->device));
    if (int rc = cfdb_check_lattice_device(m, &m->lattice)) return rc;
    m->lattice_state = m->lattice.exact ? 1 : 2;
  }
  *out = m->lattice;
  return CFDB_OK;
}

int cfdb_mesh_need_compact(cfdb_mesh* m) {
  CompactGeomDev& c = m->compact;
  if (c.ready) return CFDB_OK;
  if (int rc = cfdb_mesh_need_host_geom(m)) return rc;
  const HostGeom& g = *m->geom;
  const int64_t n = m->n, nx = m->nx, ny = m->ny, nz = m->nz;
  const int64_t yp = ny + 1, zp = nz + 4, np = (nx + 1) * yp * zp;
  auto pidx = [&](int64_t x, int64_t y, int64_t z) { return ((x + 1) * yp + (y + 1)) * zp + (z + 4); };
  std::vector<double> G(static_cast<size_t>(10 * np), 0.0);
  // face slots: +x = 5, +y = 3, +z = 1; -x = 4, -y = 2, -z = 0
  auto face = [&](int slot, int64_t i, int c3) {
    const int64_t k6 = int64_t(slot) * n + i;
    return g.normal_alt[c3 * 6 * n + k6] * g.area[k6];
  };
  const int plus_slot[3] = {5, 3, 1};
  for (int64_t x = 0; x < nx; ++x)
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t z = 0; z < nz; ++z) {
        const int64_t i = (x * ny + y) * nz + z, pi = pidx(x, y, z);
        for (int d = 0; d < 3; ++d)
          for (int c3 = 0; c3 < 3; ++c3) G[(3 * d + c3) * np + pi] = face(plus_slot[d], i, c3);
        G[9 * np + pi] = 1.0 / g.volume[i];
        // ghost neighbours below the walls: the wall face's outward vector negated
        for (int c3 = 0; c3 < 3; ++c3) {
          if (x == 0) G[(0 + c3) * np + pidx(-1, y, z)] = -face(4, i, c3);
          if (y == 0) G[(3 + c3) * np + pidx(x, -1, z)] = -face(2, i, c3);
          if (z == 0) G[(6 + c3) * np + pidx(x, y, -1)] = -face(0, i, c3);
        }
      }
  int rc = upload_as<float>(m->ctx, G.data(), int64_t(G.size()), reinterpret_cast<void**>(&c.S));
  if (rc) return rc;
  c.np = np;
  c.yp = yp;
  c.zp = zp;
  c.ready = true;
  return CFDB_OK;
}

// ---------------------------------------------------------------------------
// wave dt (host; setup-time)
// ---------------------------------------------------------------------------
extern "C" int cfdb_wave_dt(const cfdb_mesh* cm, const double* c_host, double c_const, double cfl, double* dt_out) {
  cfdb_mesh* m = const_cast<cfdb_mesh*>(cm);
  if (!m || !dt_out || !(cfl > 0)) return cfdb_fail(m ? m->ctx : nullptr, CFDB_EINVAL, "cfdb_wave_dt: bad arguments");
  if (m->uniform && !c_host) {
    if (!(c_const > 0)) return cfdb_fail(m->ctx, CFDB_EINVAL, "cfdb_wave_dt: c must be > 0");
    // 2V / sum_f c A_f = 1 / (c (1/dx + 1/dy + 1/dz)) on a uniform mesh
    const double s = (c_const / m->dx + c_const / m->dy) + c_const / m->dz;
    *dt_out = cfl / s;
    return CFDB_OK;
  }
  if (int rc = cfdb_mesh_need_host_geom(m)) return rc;
  const HostGeom& g = *m->geom;
  double best = INFINITY;
  for (int64_t i = 0; i < m->n; ++i) {
    const double c = c_host ? c_host[i] : c_const;
    if (!(c > 0)) return cfdb_fail(m->ctx, CFDB_EINVAL, "cfdb_wave_dt: c[%lld] must be > 0", (long long)i);
    double s = 0;
    for (int f = 0; f < 6; ++f) s += c * g.area[int64_t(f) * m->n + i];
    best = std::min(best, 2.0 * g.volume[i] / s);
  }
  *dt_out = cfl * best;
  return CFDB_OK;
}
