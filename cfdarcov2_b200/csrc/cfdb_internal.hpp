// Internal declarations shared by the host runtime and the kernel files of
// libcfdb.  Nothing here is part of the C ABI (include/cfdb.h).
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <functional>
#include <initializer_list>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "cfdb.h"

// ---------------------------------------------------------------------------
// Host-side geometry in double: the reference's flattened N x 6 arrays
// (entry (i, f) at f*n + i; per-dimension arrays stacked d*6n + f*n + i).
// ---------------------------------------------------------------------------
struct HostGeom {
  int64_t nx = 0, ny = 0, nz = 0, n = 0;
  std::vector<double> normal, normal_alt;  // 3 * 6n
  std::vector<double> area, alpha, len;    // 6n
  std::vector<double> volume, center, isb; // n, 3n, n
  std::vector<int64_t> ids, ibf;           // 6n
};

// Builds HostGeom (geometry.cpp).  verts may be null (uniform lattice).  mode:
// 0 reference formulas, 1 reference with component-sum areas, 2 exact vector
// areas (default of vertex meshes).  Returns false if memory runs out.
bool cfdb_build_geometry(HostGeom& g, int64_t nx, int64_t ny, int64_t nz, double dx, double dy, double dz,
                         const double* verts, int mode);

// Device copy of the geometry for the plain (per-operator) kernels in one
// precision.  ids are int32 (self on boundary faces, as the reference's _ids).
struct PlainGeomDev {
  bool ready = false;
  void* normal = nullptr;      // 3 * 6n
  void* normal_alt = nullptr;  // 3 * 6n
  void* area = nullptr;        // 6n
  void* alpha = nullptr;       // 6n
  void* len = nullptr;         // 6n
  void* volume = nullptr;      // n
  void* isb = nullptr;         // n
  void* stab_tmp = nullptr;    // 3 * 6n, allocated on first stab call
};

// Compact FP32 geometry of vertex meshes for the fused kernels: per cell the
// outward area vector of its +x/+y/+z face and 1/V (10 fields), stored on
// the lattice padded by one ghost layer below each axis (x and y) and by four
// cells below z (so the z origin of every row stays 16-byte aligned):
// cell (x, y, z) sits at ((x + 1) Yp + y + 1) Zp + z + 4 with Yp = ny + 1,
// Zp = nz + 4.  The -faces of a cell are its minus neighbours' +faces
// negated; on the -x/-y/-z walls that neighbour is a ghost entry holding the
// wall face's outward area vector negated, so no kernel needs a wall table.
// Ghost entries of the other fields are zero.
struct CompactGeomDev {
  bool ready = false;
  float* S = nullptr;  // 10 np: [Sx.x|Sx.y|Sx.z|Sy.x|...|Sz.z|1/V] over the padded lattice
  int64_t np = 0;      // padded entries per field: (nx + 1) Yp Zp
  int64_t yp = 0, zp = 0;
};

struct cfdb_ctx {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  int64_t budget = 0;
  int64_t allocated = 0;
  std::unordered_map<void*, int64_t> allocs;
  // Stream-ordered pool for per-call workspaces (checkpoint slots, adjoint
  // buffers, reduction scratch): freed blocks stay in the pool, so a repeated
  // call of the same size neither allocates nor frees device memory.
  cudaMemPool_t pool = nullptr;
  std::unordered_map<void*, int64_t> ws;
  int* d_error = nullptr;  // device error word written by bounded waits
  // Bound of the sweep kernels' mbarrier waits (SM clock cycles) and the
  // missing-copy test hook (cfdb_ctx_set_wait_limit).
  long long wait_cycles = 4000000000LL;
  int missing_plane = -1;
  cudaStream_t capture_stream = nullptr;  // private stream used to record CUDA graphs
  // Kernels launched on this context so far (graph replays count every
  // kernel node they run).
  int64_t launches = 0;
  // Instantiated step graphs of cfdb_run_steps, keyed by everything the
  // recorded launches depend on; least recently used beyond kGraphCache.
  struct GraphEntry {
    std::string key;
    cudaGraphExec_t exec = nullptr;
    int32_t chunk = 0;        // steps per replay
    int64_t per_replay = 0;   // kernels per replay
    uint64_t last_use = 0;
  };
  std::vector<GraphEntry> graphs;
  uint64_t graph_clock = 0;
  // Objects created on this context (meshes, Euler solvers, batches) with a
  // callback that detaches them when the context is destroyed first: their
  // device memory goes with the context, their own destroy then frees only
  // host memory.
  std::unordered_map<void*, std::function<void()>> children;
};

inline void cfdb_adopt(cfdb_ctx* ctx, void* child, std::function<void()> orphan) {
  if (ctx) ctx->children[child] = std::move(orphan);
}
inline void cfdb_release(cfdb_ctx* ctx, void* child) {
  if (ctx) ctx->children.erase(child);
}

// Runs `steps` calls of step(src, dst) alternating a -> b -> a ..., eagerly or
// replayed from a captured CUDA graph (graphs.cpp).  `key` names everything
// the recorded launches depend on (kernel, mesh uid, buffers, parameters); a
// graph recorded under the same key by an earlier call is replayed without
// recording again.  An empty key records a fresh graph every call.
#include <functional>
int cfdb_run_steps(cfdb_ctx* ctx, void* a, void* b, int32_t steps, int use_graph,
                   const std::function<int(const void*, void*)>& step, const std::string& key = std::string());
void cfdb_graphs_clear(cfdb_ctx* ctx);
void cfdb_jit_release(cfdb_ctx* ctx);  // unloads the context's run-time compiled modules (jit.cpp)
// Key of a cached step graph: the step kind, the mesh (by uid), dtype, path,
// the three buffers and the scalar parameters, bit for bit.
std::string graph_key(const char* kind, const struct cfdb_mesh* m, int dtype, int path, const void* a, const void* b,
                      const void* c, std::initializer_list<double> params);

struct cfdb_mesh {
  cfdb_ctx* ctx = nullptr;
  uint64_t uid = 0;  // process-unique, never reused (keys of cached step graphs)
  int64_t nx = 0, ny = 0, nz = 0, n = 0;
  double dx = 0, dy = 0, dz = 0;
  bool uniform = true;
  int geom_mode = 0;  // see cfdb_build_geometry
  std::vector<double> verts;  // vertex meshes only
  std::unique_ptr<HostGeom> geom;
  int32_t* d_ids = nullptr;
  PlainGeomDev plain[2];
  CompactGeomDev compact;
  int lattice_state = 0;  // 0 not checked, 1 exact lattice, 2 not one
  cfdb_lattice_geometry lattice{};
};

// Device ordinals the per-device caches of kernel attributes cover.
constexpr int kMaxDevices = 64;

// ---- tracing -----------------------------------------------------------------
// An NVTX range over a library call (the reference times Equation::evaluate
// with std::chrono only, examples/main_3d_heat.cpp:96-99): profilers and
// timeline tools show each run / build / gradient phase by name.  NVTX 3 is
// header-only; without a tool attached a range costs a few nanoseconds.
#include <nvtx3/nvToolsExt.h>
struct CfdbRange {
  explicit CfdbRange(const char* name) { nvtxRangePushA(name); }
  ~CfdbRange() { nvtxRangePop(); }
  CfdbRange(const CfdbRange&) = delete;
  CfdbRange& operator=(const CfdbRange&) = delete;
};

// ---- error plumbing --------------------------------------------------------
int cfdb_fail(cfdb_ctx* ctx, int code, const char* fmt, ...);
int cfdb_cuda_fail(cfdb_ctx* ctx, cudaError_t e, const char* what);
// Reads and clears the device error word (bounded waits, sweep launch
// checks); synchronises ctx->stream.  CFDB_ETIMEOUT for a wait that gave up.
int cfdb_check_device_error(cfdb_ctx* ctx);

#define CFDB_CUDA(ctx, call)                                       \
  do {                                                             \
    cudaError_t e__ = (call);                                      \
    if (e__ != cudaSuccess) return cfdb_cuda_fail((ctx), e__, #call); \
  } while (0)

// Checks for a launch error right after a kernel launch.
#define CFDB_LAUNCHED(ctx)                   \
  do {                                       \
    ++(ctx)->launches;                       \
    CFDB_CUDA(ctx, cudaGetLastError());      \
  } while (0)

// ---- memory ---------------------------------------------------------------
int cfdb_dev_alloc(cfdb_ctx* ctx, int64_t bytes, void** out);
void cfdb_dev_free(cfdb_ctx* ctx, void* p);
// Workspace from the context's pool, ordered on ctx->stream (usable by work
// enqueued after the call; freed after the work enqueued before the free).
// Counts toward the allocation budget while live.
int cfdb_ws_alloc(cfdb_ctx* ctx, int64_t bytes, void** out);
void cfdb_ws_free(cfdb_ctx* ctx, void* p);

// ---- module loading ---------------------------------------------------------
// CUDA loads a kernel at its first launch by default (lazy loading), which
// puts 0.1-1.5 ms of module work inside a caller's first step.  Each
// translation unit with kernels registers an empty anchor kernel at library
// load; context creation loads every kernel of the anchors' modules.
int cfdb_register_module(const void* anchor_kernel);
#define CFDB_MODULE_ANCHOR                                                                      \
  namespace {                                                                                   \
  __global__ void cfdb_module_anchor_k() {}                                                     \
  const int cfdb_module_anchor_reg_ = cfdb_register_module(reinterpret_cast<const void*>(&cfdb_module_anchor_k)); \
  }

// ---- geometry helpers ------------------------------------------------------
int cfdb_mesh_need_host_geom(cfdb_mesh* m);
int cfdb_mesh_need_plain(cfdb_mesh* m, int dtype);
// fills the plain arrays of dtype on the device (geometry_dev.cu)
int cfdb_build_plain_device(cfdb_mesh* m, int dtype, PlainGeomDev& p);
// samples and checks the lattice constants on the device (geometry_dev.cu)
int cfdb_check_lattice_device(cfdb_mesh* m, cfdb_lattice_geometry* out);
int cfdb_mesh_need_compact(cfdb_mesh* m);

inline size_t dtype_size(int dtype) { return dtype == CFDB_F64 ? 8 : 4; }
inline bool dtype_ok(int dtype) { return dtype == CFDB_F32 || dtype == CFDB_F64; }

int cfdb_check_mesh(cfdb_ctx* ctx, cfdb_mesh* m);
void cfdb_mesh_orphan(cfdb_mesh* m);

// ---- launchers implemented in the kernel files ------------------------------
// plain_ops.cu
int plain_lapl(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* phi, void* out, int mask);
int plain_heat_update(cfdb_ctx* ctx, int dtype, const void* L, const void* T, double k, double dt, void* Tn,
                      int64_t n);
int plain_wave_step(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* q, void* qn, const void* c,
                    double cconst, int mode, double dt);
int plain_wave_adjoint(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* q, const void* lam1, void* lam0,
                       const void* c, void* gc, double dt);
// fused_tma.cu
int fused_heat_step(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* T, void* Tn, double k, double dt,
                    const void* fixed = nullptr);
int fused_d2t_step(cfdb_ctx* ctx, cfdb_mesh* m, const void* u, const void* u_prev, void* u_next, double k,
                   const int32_t* masks, int32_t n_terms, double dt, int first_step);
// All `steps` FP32 heat steps in one thread-block-cluster launch with the
// field resident in distributed shared memory (resident.cu); CFDB_EUNSUPPORTED
// when the mesh does not fit (nothing launched).
int heat_resident_run(cfdb_ctx* ctx, cfdb_mesh* m, const void* Ta, void* Tb, double k, double dt, int32_t steps,
                      int* launched);
int fused_wave_step(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* q, void* qn, const void* c,
                    double cconst, int mode, double dt);
// distorted.cu
int compact_wave_step(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* q, void* qn, const void* c,
                      double cconst, int mode, double dt);
// adjoint.cu
int fused_wave_adjoint(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* q, const void* lam1, void* lam0,
                       const void* c, void* gc, double dt);

// Shared launch-size helper: a grid-stride grid of at most `per_sm` CTAs per SM.
inline int grid_for(const cfdb_ctx* ctx, int64_t n, int threads, int per_sm = 8) {
  int64_t want = (n + threads - 1) / threads;
  int64_t cap = int64_t(ctx->num_sms > 0 ? ctx->num_sms : 148) * per_sm;
  if (want > cap) want = cap;
  if (want < 1) want = 1;
  return int(want);
}
