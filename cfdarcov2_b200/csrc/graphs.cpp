// Multi-step runs with CUDA-graph replay.  The step launches of a run are
// recorded once on a private stream (so the caller's stream may be the legacy
// default stream, which cannot be captured) and the instantiated graph is
// launched on the caller's stream chunk after chunk.
#include <algorithm>

#include "cfdb_internal.hpp"

int cfdb_run_steps(cfdb_ctx* ctx, void* a, void* b, int32_t steps, int use_graph,
                   const std::function<int(const void*, void*)>& step, int64_t* launches) {
  if (steps < 0) return cfdb_fail(ctx, CFDB_EINVAL, "steps must be >= 0");
  auto one = [&](int32_t k) { return (k & 1) ? step(b, a) : step(a, b); };
  int32_t k = 0;
  const int32_t eager = use_graph ? std::min<int32_t>(steps, 2) : steps;
  for (; k < eager; ++k)
    if (int rc = one(k)) return rc;
  if (launches) *launches = eager;
  if (k >= steps) return CFDB_OK;
  // record an even chunk of steps (so every replay starts from buffer a)
  const int32_t chunk = std::max<int32_t>(2, std::min<int32_t>(64, (steps - k) & ~1));
  if (!ctx->capture_stream)
    CFDB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->capture_stream, cudaStreamNonBlocking));
  cudaStream_t user = ctx->stream;
  ctx->stream = ctx->capture_stream;
  cudaGraph_t graph = nullptr;
  int rc = CFDB_OK;
  cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    for (int32_t j = 0; j < chunk && !rc; ++j) rc = one(j);
    cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &graph);
    if (!rc && e2 != cudaSuccess) rc = cfdb_cuda_fail(ctx, e2, "cudaStreamEndCapture");
  } else {
    rc = cfdb_cuda_fail(ctx, e, "cudaStreamBeginCapture");
  }
  ctx->stream = user;
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return cfdb_cuda_fail(ctx, e, "cudaGraphInstantiate");
  // k is even here (eager == 2), so buffer parity is preserved
  const int32_t reps = (steps - k) / chunk;
  for (int32_t r = 0; r < reps && !rc; ++r) {
    e = cudaGraphLaunch(exec, ctx->stream);
    if (e != cudaSuccess) rc = cfdb_cuda_fail(ctx, e, "cudaGraphLaunch");
  }
  k += reps * chunk;
  if (launches) *launches += int64_t(reps) * chunk;
  cudaGraphExecDestroy(exec);
  for (; k < steps && !rc; ++k) {
    rc = one(k);
    if (!rc && launches) ++*launches;
  }
  return rc;
}
