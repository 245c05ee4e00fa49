// Multi-step runs with CUDA-graph replay.  The step launches of a run are
// recorded once on a private stream (so the caller's stream may be the legacy
// default stream, which cannot be captured) and the instantiated graph is
// launched on the caller's stream chunk after chunk.  Instantiated graphs are
// cached on the context under a key naming everything the recorded launches
// depend on, so a repeated run (the same mesh, buffers and parameters) pays
// neither the recording nor the instantiation again: the device never waits
// for the host between runs.
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "cfdb_internal.hpp"

namespace {

constexpr size_t kGraphCache = 8;

cfdb_ctx::GraphEntry* find_graph(cfdb_ctx* ctx, const std::string& key, int32_t chunk) {
  for (auto& g : ctx->graphs)
    if (g.chunk == chunk && g.key == key) return &g;
  return nullptr;
}

void store_graph(cfdb_ctx* ctx, cfdb_ctx::GraphEntry entry) {
  if (ctx->graphs.size() >= kGraphCache) {
    auto lru = std::min_element(ctx->graphs.begin(), ctx->graphs.end(),
                                [](const auto& x, const auto& y) { return x.last_use < y.last_use; });
    cudaGraphExecDestroy(lru->exec);
    ctx->graphs.erase(lru);
  }
  ctx->graphs.push_back(std::move(entry));
}

}  // namespace

std::string graph_key(const char* kind, const cfdb_mesh* m, int dtype, int path, const void* a, const void* b,
                      const void* c, std::initializer_list<double> params) {
  std::string k(kind);
  char buf[96];
  snprintf(buf, sizeof(buf), "|%llu|%d|%d|%p|%p|%p", (unsigned long long)m->uid, dtype, path, a, b, c);
  k += buf;
  for (double p : params) {
    uint64_t bits;
    std::memcpy(&bits, &p, sizeof(bits));
    snprintf(buf, sizeof(buf), "|%016llx", (unsigned long long)bits);
    k += buf;
  }
  return k;
}

void cfdb_graphs_clear(cfdb_ctx* ctx) {
  for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.exec);
  ctx->graphs.clear();
}

int cfdb_run_steps(cfdb_ctx* ctx, void* a, void* b, int32_t steps, int use_graph,
                   const std::function<int(const void*, void*)>& step, const std::string& key) {
  if (steps < 0) return cfdb_fail(ctx, CFDB_EINVAL, "steps must be >= 0");
  auto one = [&](int32_t k) { return (k & 1) ? step(b, a) : step(a, b); };
  int32_t k = 0;
  // an even chunk of steps per replay (so every replay starts from buffer a)
  const int32_t chunk = std::max<int32_t>(2, std::min<int32_t>(64, (steps - std::min(steps, 2)) & ~1));
  cfdb_ctx::GraphEntry* cached = (use_graph && !key.empty()) ? find_graph(ctx, key, chunk) : nullptr;
  // without a cached graph, two eager steps first perform any one-time setup
  const int32_t eager = use_graph ? (cached ? 0 : std::min<int32_t>(steps, 2)) : steps;
  for (; k < eager; ++k)
    if (int rc = one(k)) return rc;
  if (k >= steps) return CFDB_OK;
  if (steps - k < chunk) {  // fewer steps than one replay
    for (; k < steps; ++k)
      if (int rc = one(k)) return rc;
    return CFDB_OK;
  }
  cudaGraphExec_t exec = nullptr;
  int64_t per_replay = 0;
  if (cached) {
    exec = cached->exec;
    per_replay = cached->per_replay;
    cached->last_use = ++ctx->graph_clock;
  } else {
    if (!ctx->capture_stream)
      CFDB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->capture_stream, cudaStreamNonBlocking));
    cudaStream_t user = ctx->stream;
    ctx->stream = ctx->capture_stream;
    const int64_t before = ctx->launches;  // recorded launches run only when replayed
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
    per_replay = ctx->launches - before;
    ctx->launches = before;
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cfdb_cuda_fail(ctx, e, "cudaGraphInstantiate");
    if (!key.empty()) {
      cfdb_ctx::GraphEntry entry;
      entry.key = key;
      entry.exec = exec;
      entry.chunk = chunk;
      entry.per_replay = per_replay;
      entry.last_use = ++ctx->graph_clock;
      store_graph(ctx, std::move(entry));
    }
  }
  // k is even here (0 or 2), so buffer parity is preserved
  const int32_t reps = (steps - k) / chunk;
  int rc = CFDB_OK;
  for (int32_t r = 0; r < reps && !rc; ++r) {
    cudaError_t e = cudaGraphLaunch(exec, ctx->stream);
    if (e != cudaSuccess) rc = cfdb_cuda_fail(ctx, e, "cudaGraphLaunch");
    else ctx->launches += per_replay;
  }
  k += reps * chunk;
  if (key.empty()) cudaGraphExecDestroy(exec);
  for (; k < steps && !rc; ++k) rc = one(k);
  return rc;
}
