// Host side of the TMA stencil sweep: tensor-map encoding through the driver
// entry point (no libcuda link), tile/chunk selection and the launch.
#pragma once
#include <atomic>

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "cfdb_internal.hpp"
#include "tma_stencil.cuh"

namespace stencil {

inline PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// 4-D map over a float32 state of nf fields stored field after field:
// dims (z, y, x, field), box (TZ+8, TY+2, 1, nf).
inline int encode_state(cfdb_ctx* ctx, CUtensorMap* map, const void* base, const cfdb_mesh* m, int nf, int tz,
                        int ty) {
  auto fn = encode_fn();
  if (!fn) return cfdb_fail(ctx, CFDB_ECUDA, "cuTensorMapEncodeTiled entry point unavailable");
  cuuint64_t dims[4] = {cuuint64_t(m->nz), cuuint64_t(m->ny), cuuint64_t(m->nx), cuuint64_t(nf)};
  cuuint64_t strides[3] = {cuuint64_t(m->nz) * 4, cuuint64_t(m->nz * m->ny) * 4, cuuint64_t(m->n) * 4};
  cuuint32_t box[4] = {cuuint32_t(tz + 8), cuuint32_t(ty + 2), 1, cuuint32_t(nf)};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void*>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cfdb_fail(ctx, CFDB_ECUDA, "cuTensorMapEncodeTiled (state) failed with %d", int(r));
  return CFDB_OK;
}

// 3-D map over one float32 field: dims (z, y, x), box (TZ+8, TY+2, 1).
inline int encode_field(cfdb_ctx* ctx, CUtensorMap* map, const void* base, const cfdb_mesh* m, int tz, int ty) {
  auto fn = encode_fn();
  if (!fn) return cfdb_fail(ctx, CFDB_ECUDA, "cuTensorMapEncodeTiled entry point unavailable");
  cuuint64_t dims[3] = {cuuint64_t(m->nz), cuuint64_t(m->ny), cuuint64_t(m->nx)};
  cuuint64_t strides[2] = {cuuint64_t(m->nz) * 4, cuuint64_t(m->nz * m->ny) * 4};
  cuuint32_t box[3] = {cuuint32_t(tz + 8), cuuint32_t(ty + 2), 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cfdb_fail(ctx, CFDB_ECUDA, "cuTensorMapEncodeTiled (field) failed with %d", int(r));
  return CFDB_OK;
}

// Checks the layout requirements of the sweep.
inline int check_sweep(cfdb_ctx* ctx, const cfdb_mesh* m, std::initializer_list<const void*> ptrs) {
  if (!m->uniform) return cfdb_fail(ctx, CFDB_EUNSUPPORTED, "the TMA sweep needs a uniform (structured) mesh");
  if (m->nz % 4 != 0)
    return cfdb_fail(ctx, CFDB_EUNSUPPORTED,
                     "the TMA sweep needs nz %% 4 == 0 (16-byte rows); nz = %lld: use CFDB_PATH_PLAIN",
                     (long long)m->nz);
  if (m->nx > 2147483647LL / 2) return cfdb_fail(ctx, CFDB_EUNSUPPORTED, "mesh too large for int32 TMA coordinates");
  for (const void* p : ptrs)
    if (p && (reinterpret_cast<uintptr_t>(p) & 15u))
      return cfdb_fail(ctx, CFDB_EINVAL, "the TMA sweep needs 16-byte aligned field pointers");
  return CFDB_OK;
}

struct SweepShape {
  int tiles, chunks;
};

// Grid of tiles x chunks CTAs.  resident = CTAs of this kernel one SM holds
// (occupancy API).  The x axis is cut into as many chunks as fill the
// resident slots of all SMs in one wave (chunk lengths differ by at most one
// plane, so every CTA finishes at about the same time); when the tiles alone
// exceed one wave the grid keeps one chunk per tile.
inline SweepShape sweep_shape(const cfdb_ctx* ctx, const cfdb_mesh* m, int tz, int ty, int resident) {
  SweepShape s;
  s.tiles = int(((m->nz + tz - 1) / tz) * ((m->ny + ty - 1) / ty));
  const int slots = std::max(1, ctx->num_sms) * std::max(1, resident);
  int chunks = std::max(1, slots / s.tiles);
  chunks = int(std::min<int64_t>(chunks, m->nx));
  s.chunks = std::min(chunks, 65535);
  return s;
}

// Launches one sweep: q holds the NF state fields, aux the NA auxiliary
// fields (may be NULL when NA == 0), c the coefficient field (HAS_C), out
// receives the NF new state fields.
template <class Phys, int TZ, int TY, int S, int VZ = 4>
int launch_sweep(cfdb_ctx* ctx, const cfdb_mesh* m, const void* q, const void* aux, const void* c, void* out,
                 const typename Phys::Params& prm, int ctas_per_sm, int* launched_grid = nullptr) {
  using L = Layout<TZ, TY, S, Phys::NF, Phys::NA, Phys::HAS_C, VZ>;
  static_assert(TZ % VZ == 0 && (VZ == 1 || VZ == 2 || VZ == 4), "bad vector width");
  CUtensorMap tq, ta, tc;
  if (int rc = encode_state(ctx, &tq, q, m, Phys::NF, TZ, TY)) return rc;
  ta = tq;
  tc = tq;
  if constexpr (Phys::NA > 0) {
    if (int rc = encode_state(ctx, &ta, aux, m, Phys::NA, TZ, TY)) return rc;
  }
  if constexpr (Phys::HAS_C) {
    if (int rc = encode_field(ctx, &tc, c, m, TZ, TY)) return rc;
  }
  auto kern = sweep_kernel<Phys, TZ, TY, S, VZ>;
  // the shared-memory attribute is a per-device setting: set it (and measure
  // the occupancy) once per device and kernel instantiation
  static std::atomic<int> resident_of[kMaxDevices] = {};
  if (ctx->device < 0 || ctx->device >= kMaxDevices)
    return cfdb_fail(ctx, CFDB_EUNSUPPORTED, "device ordinal %d beyond %d", ctx->device, kMaxDevices);
  int resident = resident_of[ctx->device].load(std::memory_order_acquire);
  if (!resident) {
    CFDB_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(L::SMEM_BYTES)));
    CFDB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kern, L::THREADS, L::SMEM_BYTES));
    if (resident < 1) return cfdb_fail(ctx, CFDB_EUNSUPPORTED, "sweep kernel does not fit on an SM");
    resident_of[ctx->device].store(resident, std::memory_order_release);
  }
  const SweepShape sh = sweep_shape(ctx, m, TZ, TY, ctas_per_sm > 0 ? std::min(ctas_per_sm, resident) : resident);
  Geometry g{int(m->nx), int(m->ny), int(m->nz), sh.chunks, (long long)m->n, ctx->wait_cycles, ctx->missing_plane};
  // Programmatic stream serialisation: the CTAs of this step may become
  // resident while the previous kernel drains; the kernel waits for it
  // (griddepcontrol.wait) before touching global memory.
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(sh.tiles, sh.chunks);
  cfg.blockDim = dim3(L::THREADS);
  cfg.dynamicSmemBytes = L::SMEM_BYTES;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CFDB_CUDA(ctx, cudaLaunchKernelEx(&cfg, kern, tq, ta, tc, g, static_cast<float*>(out), prm, ctx->d_error));
  ++ctx->launches;
  if (launched_grid) *launched_grid = sh.tiles * sh.chunks;
  return CFDB_OK;
}

}  // namespace stencil

#include "face_sweep.cuh"

namespace stencil {

// 4-D map over nf float32 fields stored field after field on a (zp, yp, xp)
// lattice of np entries per field, box (bz, by, 1, nf): one plane and all
// fields per copy.
inline int encode_box(cfdb_ctx* ctx, CUtensorMap* map, const void* base, int64_t zp, int64_t yp, int64_t xp,
                      int64_t np, int nf, int bz, int by) {
  auto fn = encode_fn();
  if (!fn) return cfdb_fail(ctx, CFDB_ECUDA, "cuTensorMapEncodeTiled entry point unavailable");
  cuuint64_t dims[4] = {cuuint64_t(zp), cuuint64_t(yp), cuuint64_t(xp), cuuint64_t(nf)};
  cuuint64_t strides[3] = {cuuint64_t(zp) * 4, cuuint64_t(zp * yp) * 4, cuuint64_t(np) * 4};
  cuuint32_t box[4] = {cuuint32_t(bz), cuuint32_t(by), 1, cuuint32_t(nf)};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void*>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cfdb_fail(ctx, CFDB_ECUDA, "cuTensorMapEncodeTiled (box) failed with %d", int(r));
  return CFDB_OK;
}

// Launches one face-flux sweep (face_sweep.cuh): q holds the NF state
// fields, pg the NG per-cell geometry fields on the padded lattice (unused
// when NG == 0), out receives the NF new state fields.  Grid and launch as
// launch_sweep.
template <class Phys, int TZ, int TY, int S, int VZ>
int launch_face_sweep(cfdb_ctx* ctx, const cfdb_mesh* m, const void* q, const PaddedGeom& pg, void* out,
                      const typename Phys::Params& prm, int ctas_per_sm, int* launched_grid = nullptr) {
  using L = FaceLayout<TZ, TY, S, Phys::NF, Phys::NG, Phys::ND, VZ>;
  static_assert(TZ % VZ == 0 && (VZ == 1 || VZ == 2 || VZ == 4), "bad vector width");
  static_assert(TZ % 4 == 0, "z tiles must keep 16-byte aligned origins");
  CUtensorMap tq, tg;
  if (int rc = encode_box(ctx, &tq, q, m->nz, m->ny, m->nx, m->n, Phys::NF, TZ + 8, TY + 2)) return rc;
  tg = tq;
  if constexpr (Phys::NG > 0) {
    if (pg.zp != m->nz + 4 || pg.yp != m->ny + 1 || pg.xp != m->nx + 1 || pg.np != pg.zp * pg.yp * pg.xp ||
        (reinterpret_cast<uintptr_t>(pg.base) & 15u))
      return cfdb_fail(ctx, CFDB_EINVAL, "face sweep: geometry is not on the padded lattice of the mesh");
    if (int rc = encode_box(ctx, &tg, pg.base, pg.zp, pg.yp, pg.xp, pg.np, Phys::NG, TZ + 4, TY + 1)) return rc;
  }
  auto kern = face_sweep_kernel<Phys, TZ, TY, S, VZ>;
  static std::atomic<int> resident_of[kMaxDevices] = {};
  if (ctx->device < 0 || ctx->device >= kMaxDevices)
    return cfdb_fail(ctx, CFDB_EUNSUPPORTED, "device ordinal %d beyond %d", ctx->device, kMaxDevices);
  int resident = resident_of[ctx->device].load(std::memory_order_acquire);
  if (!resident) {
    CFDB_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(L::SMEM_BYTES)));
    CFDB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kern, L::THREADS, L::SMEM_BYTES));
    if (resident < 1) return cfdb_fail(ctx, CFDB_EUNSUPPORTED, "face sweep kernel does not fit on an SM");
    resident_of[ctx->device].store(resident, std::memory_order_release);
  }
  const SweepShape sh = sweep_shape(ctx, m, TZ, TY, ctas_per_sm > 0 ? std::min(ctas_per_sm, resident) : resident);
  Geometry g{int(m->nx), int(m->ny), int(m->nz), sh.chunks, (long long)m->n, ctx->wait_cycles, ctx->missing_plane};
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(sh.tiles, sh.chunks);
  cfg.blockDim = dim3(L::THREADS);
  cfg.dynamicSmemBytes = L::SMEM_BYTES;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CFDB_CUDA(ctx, cudaLaunchKernelEx(&cfg, kern, tq, tg, g, static_cast<float*>(out), prm, ctx->d_error));
  ++ctx->launches;
  if (launched_grid) *launched_grid = sh.tiles * sh.chunks;
  return CFDB_OK;
}

}  // namespace stencil
