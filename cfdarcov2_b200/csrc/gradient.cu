// Gradient of J = 0.5 |p_T - p_target|^2 with respect to the sound-speed
// field c and the initial pressure p0, through the discrete adjoint of the
// acoustic step (speed_mode 1).  With snapshots >= steps every forward state
// is written straight into its own slot (the forward step's output IS the
// checkpoint: no copies) and the reverse sweep reads them back; with fewer
// slots the binomial schedule of revolve.cpp recomputes the missing states.
#include <algorithm>
#include <cmath>
#include <vector>

#include "cfdb_internal.hpp"

CFDB_MODULE_ANCHOR

int cfdb_revolve_build(int32_t steps, int32_t snapshots, std::vector<int32_t>& act, std::vector<int32_t>& arg,
                       std::vector<int32_t>& at, int64_t* forward);

namespace {

constexpr int kThreads = 256;

template <class R>
__global__ void init_adjoint_k(const R* __restrict__ qT, const R* __restrict__ target, R* __restrict__ lam, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    lam[i] = qT[i] - target[i];
    lam[n + i] = R(0);
    lam[2 * n + i] = R(0);
    lam[3 * n + i] = R(0);
  }
}

template <class R>
__global__ void misfit_k(const R* __restrict__ qT, const R* __restrict__ target, long long n, double* __restrict__ part) {
  __shared__ double red[kThreads / 32];
  double s = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double d = double(qT[i]) - double(target[i]);
    s += d * d;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < int(blockDim.x / 32); ++w) t += red[w];
    part[blockIdx.x] = t;
  }
}

__global__ void misfit_final_k(const double* __restrict__ part, int np, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double t = 0;
    for (int k = 0; k < np; ++k) t += part[k];
    out[0] = 0.5 * t;
  }
}

struct Run {
  cfdb_ctx* ctx;
  cfdb_mesh* m;
  int dtype, path;
  const void* c;
  double dt;
  size_t esz;
  int64_t n;

  int step(const void* src, void* dst) const {
    return cfdb_wave_step(ctx, m, dtype, path, src, dst, c, 0.0, 1, dt);
  }
  int adjoint(const void* q, const void* lam1, void* lam0, void* gc) const {
    return cfdb_wave_adjoint_step(ctx, m, dtype, path, q, lam1, lam0, c, gc, dt);
  }
  int copy(void* dst, const void* src) const {
    CFDB_CUDA(ctx, cudaMemcpyAsync(dst, src, 4 * n * esz, cudaMemcpyDeviceToDevice, ctx->stream));
    return CFDB_OK;
  }
  // J into *host (synchronous) and, when lam != nullptr, the adjoint seed.
  int misfit(const void* qT, const void* target, void* lam, double* host, void* scratch) const {
    const int grid = grid_for(ctx, n, kThreads, 2);
    double* part = static_cast<double*>(scratch);
    double* res = part + grid;
    if (dtype == CFDB_F64) {
      misfit_k<double><<<grid, kThreads, 0, ctx->stream>>>((const double*)qT, (const double*)target, n, part);
      if (lam) init_adjoint_k<double><<<grid_for(ctx, n, kThreads), kThreads, 0, ctx->stream>>>((const double*)qT, (const double*)target, (double*)lam, n);
    } else {
      misfit_k<float><<<grid, kThreads, 0, ctx->stream>>>((const float*)qT, (const float*)target, n, part);
      if (lam) init_adjoint_k<float><<<grid_for(ctx, n, kThreads), kThreads, 0, ctx->stream>>>((const float*)qT, (const float*)target, (float*)lam, n);
    }
    misfit_final_k<<<1, 32, 0, ctx->stream>>>(part, grid, res);
    CFDB_LAUNCHED(ctx);
    CFDB_CUDA(ctx, cudaMemcpyAsync(host, res, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return CFDB_OK;
  }
};

int check_args(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, int path, const void* q0, const void* c, const void* target,
               int32_t steps, double dt, const char* fn) {
  if (int rc = cfdb_check_mesh(ctx, m)) return rc;
  if (!dtype_ok(dtype)) return cfdb_fail(ctx, CFDB_EINVAL, "%s: unknown dtype %d", fn, dtype);
  if (path != CFDB_PATH_PLAIN && path != CFDB_PATH_FUSED) return cfdb_fail(ctx, CFDB_EINVAL, "%s: unknown path", fn);
  if (!q0 || !c || !target) return cfdb_fail(ctx, CFDB_EINVAL, "%s: NULL input", fn);
  if (steps < 1 || !(dt > 0) || !std::isfinite(dt)) return cfdb_fail(ctx, CFDB_EINVAL, "%s: need steps >= 1 and dt > 0", fn);
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  return CFDB_OK;
}

// Workspaces of one call, taken from the context's pool and returned to it
// (stream-ordered) when the call ends.
struct Bufs {
  cfdb_ctx* ctx;
  std::vector<void*> v;
  ~Bufs() {
    for (void* p : v) cfdb_ws_free(ctx, p);
  }
  int get(int64_t bytes, void** out) {
    int rc = cfdb_ws_alloc(ctx, bytes, out);
    if (!rc) v.push_back(*out);
    return rc;
  }
};

}  // namespace

extern "C" int cfdb_wave_objective(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, int path, const void* q0, const void* c,
                                   const void* target, int32_t steps, double dt, double* J_out) {
  CfdbRange range_("cfdb_wave_objective");
  if (int rc = check_args(ctx, m, dtype, path, q0, c, target, steps, dt, "cfdb_wave_objective")) return rc;
  if (!J_out) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_wave_objective: J_out is NULL");
  Run R{ctx, m, dtype, path, c, dt, dtype_size(dtype), m->n};
  Bufs B{ctx, {}};
  void *a, *b, *scratch;
  if (int rc = B.get(int64_t(4 * R.esz) * R.n, &a)) return rc;
  if (int rc = B.get(int64_t(4 * R.esz) * R.n, &b)) return rc;
  if (int rc = B.get(int64_t(8) * (grid_for(ctx, R.n, kThreads, 2) + 2), &scratch)) return rc;
  if (int rc = R.copy(a, q0)) return rc;
  if (int rc = cfdb_run_steps(ctx, a, b, steps, 1, [&](const void* s, void* d) { return R.step(s, d); },
                              graph_key("wave", m, dtype, path, a, b, c, {0.0, 1.0, dt})))
    return rc;
  return R.misfit((steps & 1) ? b : a, target, nullptr, J_out, scratch);
}

extern "C" int cfdb_wave_gradient(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, int path, const void* q0, const void* c,
                                  const void* target, int32_t steps, double dt, int32_t snapshots, double* J_out,
                                  void* grad_c, void* grad_p0, cfdb_gradient_stats* stats) {
  CfdbRange range_("cfdb_wave_gradient");
  if (int rc = check_args(ctx, m, dtype, path, q0, c, target, steps, dt, "cfdb_wave_gradient")) return rc;
  if (!J_out || !grad_c || !grad_p0) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_wave_gradient: NULL output");
  if (snapshots < 1) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_wave_gradient: snapshots must be >= 1");
  Run R{ctx, m, dtype, path, c, dt, dtype_size(dtype), m->n};
  const int64_t sb = int64_t(4 * R.esz) * R.n;  // one state
  Bufs B{ctx, {}};
  void *lamA, *lamB, *scratch;
  if (int rc = B.get(sb, &lamA)) return rc;
  if (int rc = B.get(sb, &lamB)) return rc;
  if (int rc = B.get(int64_t(8) * (grid_for(ctx, R.n, kThreads, 2) + 2), &scratch)) return rc;
  CFDB_CUDA(ctx, cudaMemsetAsync(grad_c, 0, R.esz * R.n, ctx->stream));
  cudaEvent_t e0, e1, e2;
  CFDB_CUDA(ctx, cudaEventCreate(&e0));
  CFDB_CUDA(ctx, cudaEventCreate(&e1));
  CFDB_CUDA(ctx, cudaEventCreate(&e2));
  struct EvGuard {
    cudaEvent_t a, b, c;
    ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); cudaEventDestroy(c); }
  } evg{e0, e1, e2};
  cfdb_gradient_stats st{};
  int rc = CFDB_OK;
  void* lam = lamA;
  void* lam_next = lamB;
  auto adj = [&](const void* q) {
    int r = R.adjoint(q, lam, lam_next, grad_c);
    std::swap(lam, lam_next);
    ++st.adjoint_steps;
    return r;
  };

  if (snapshots >= steps) {
    // every state in its own slot; the forward step writes the checkpoint
    char* states = nullptr;
    if ((rc = B.get(sb * (int64_t(steps) + 1), reinterpret_cast<void**>(&states))))
      return cfdb_fail(ctx, rc, "cfdb_wave_gradient: %d stored states (%lld bytes) do not fit; pass fewer snapshots",
                       steps + 1, (long long)(sb * (int64_t(steps) + 1)));
    auto slot = [&](int t) { return static_cast<void*>(states + sb * int64_t(t)); };
    if ((rc = R.copy(slot(0), q0))) return rc;
    cudaEventRecord(e0, ctx->stream);
    {
      CfdbRange forward("cfdb_wave_gradient: forward sweep");
      for (int t = 0; t < steps && !rc; ++t) rc = R.step(slot(t), slot(t + 1));
    }
    cudaEventRecord(e1, ctx->stream);
    if (rc) return rc;
    st.forward_steps = steps;
    st.snapshots_used = steps + 1;
    if ((rc = R.misfit(slot(steps), target, lam, J_out, scratch))) return rc;
    CfdbRange reverse("cfdb_wave_gradient: reverse sweep");
    for (int t = steps - 1; t >= 0 && !rc; --t) rc = adj(slot(t));
  } else {
    std::vector<int32_t> act, arg, at;
    int64_t fwd = 0;
    cfdb_revolve_build(steps, snapshots, act, arg, at, &fwd);
    char* slots = nullptr;
    void *cur, *tmp;
    if ((rc = B.get(sb * snapshots, reinterpret_cast<void**>(&slots)))) return rc;
    if ((rc = B.get(sb, &cur))) return rc;
    if ((rc = B.get(sb, &tmp))) return rc;
    auto slot = [&](int k) { return static_cast<void*>(slots + sb * int64_t(k)); };
    if ((rc = R.copy(cur, q0))) return rc;
    cudaEventRecord(e0, ctx->stream);
    bool first_turn_seen = false;
    for (size_t k = 0; k < act.size() && !rc; ++k) {
      switch (act[k]) {
        case CFDB_RV_TAKESHOT: rc = R.copy(slot(arg[k]), cur); break;
        case CFDB_RV_RESTORE: rc = R.copy(cur, slot(arg[k])); break;
        case CFDB_RV_ADVANCE:
          for (int j = 0; j < arg[k] && !rc; ++j) {
            rc = R.step(cur, tmp);
            std::swap(cur, tmp);
            ++st.forward_steps;
          }
          break;
        case CFDB_RV_FIRSTURN:
          cudaEventRecord(e1, ctx->stream);
          first_turn_seen = true;
          if ((rc = R.step(cur, tmp))) break;  // q_T
          ++st.forward_steps;
          if ((rc = R.misfit(tmp, target, lam, J_out, scratch))) break;
          rc = adj(cur);
          break;
        case CFDB_RV_YOUTURN: rc = adj(cur); break;
        default: rc = cfdb_fail(ctx, CFDB_EINVAL, "corrupt checkpoint schedule"); break;
      }
    }
    if (!first_turn_seen && !rc) rc = cfdb_fail(ctx, CFDB_EINVAL, "checkpoint schedule has no first turn");
    st.snapshots_used = snapshots;
  }
  if (rc) return rc;
  // dJ/dp0 = the pressure block of lam_0
  CFDB_CUDA(ctx, cudaMemcpyAsync(grad_p0, lam, R.esz * R.n, cudaMemcpyDeviceToDevice, ctx->stream));
  cudaEventRecord(e2, ctx->stream);
  CFDB_CUDA(ctx, cudaEventSynchronize(e2));
  float f = 0, r = 0;
  cudaEventElapsedTime(&f, e0, e1);
  cudaEventElapsedTime(&r, e1, e2);
  st.forward_ms = f;
  st.reverse_ms = r;
  if (stats) *stats = st;
  return CFDB_OK;
}
