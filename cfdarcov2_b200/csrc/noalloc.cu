// Allocation-free variant of the FP64 compensated total (cfdb_total_fp64).
//
// Some callers cannot allocate device memory at all: a plugin living inside a
// host application that owns every device allocation through its own pool,
// a step recorded into someone else's CUDA graph, or a real-time loop that
// cannot afford the implicit synchronisation of cudaMalloc/cudaFree.  They
// still own their input field and their output slot; what they cannot provide
// is the per-CTA scratch the reduction needs.  This file keeps that scratch in
// a file-scope __device__ array instead, so the entry point calls no
// cudaMalloc, cudaFree or any allocating library routine.
//
// Limits and sharing rules:
//  * at most kMaxChunks * kChunk = 268,435,456 cells per call (1 MiB of
//    scratch, held by every GPU that loads the library until the process
//    exits); larger n is rejected with CFDB_EINVAL before anything is launched;
//  * every call overwrites all the scratch it reads (one partial per chunk and
//    the result slot), so nothing has to be cleared between calls;
//  * all calls share the one array: calls that overlap on the GPU (different
//    streams, or different host threads on the same device) race and must be
//    serialised by the caller;
//  * the first call on a device resolves the array's device address with
//    cudaGetSymbolAddress (host code cannot pass the array's name to a kernel:
//    on the host it is only a stand-in, not a device address); make that first
//    call outside any stream capture.  The address is cached per device for
//    the life of the process: after cudaDeviceReset (which unloads the
//    library's device code) the library must be unloaded and loaded again
//    before this entry point is used on that device.
#include <cmath>
#include <mutex>

#include "cfdb_internal.hpp"

CFDB_MODULE_ANCHOR

namespace {

constexpr int kChunk = 4096;             // cells reduced by one CTA
constexpr long long kMaxChunks = 65536;  // scratch partials
constexpr int kThreads = 256;

struct Pair {
  double s, c;  // Neumaier running sum and compensation
};

// partials [0, kMaxChunks) and the result slot kMaxChunks
static __device__ __align__(256) Pair g_noalloc_scratch[kMaxChunks + 1];

__device__ __forceinline__ void pair_add(Pair& a, double x) {
  const double t = a.s + x;
  if (fabs(a.s) >= fabs(x)) a.c += (a.s - t) + x; else a.c += (x - t) + a.s;
  a.s = t;
}

template <class R>
__global__ void chunk_total_k(const R* __restrict__ f, const R* __restrict__ vol, double vconst, long long n,
                              Pair* __restrict__ part) {
  __shared__ Pair red[kThreads / 32];
  const long long begin = (long long)blockIdx.x * kChunk;
  const long long end = min(n, begin + kChunk);
  Pair a{0.0, 0.0};
  for (long long i = begin + threadIdx.x; i < end; i += blockDim.x)
    pair_add(a, double(f[i]) * (vol ? double(vol[i]) : vconst));
  for (int o = 16; o > 0; o >>= 1) {
    const double s = __shfl_xor_sync(0xffffffffu, a.s, o);
    const double c = __shfl_xor_sync(0xffffffffu, a.c, o);
    pair_add(a, s);
    a.c += c;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    Pair t{0.0, 0.0};
    for (int w = 0; w < kThreads / 32; ++w) {
      pair_add(t, red[w].s);
      t.c += red[w].c;
    }
    part[blockIdx.x] = t;
  }
}

// One warp: lane l folds partials l, l + 32, l + 64, ... (coalesced loads,
// at most 2048 dependent adds per lane at the maximum size), then the lanes
// merge pairwise through shuffles in a fixed order, so the result does not
// depend on timing.
__global__ void chunk_final_k(const Pair* __restrict__ part, int np, Pair* __restrict__ slot, double* __restrict__ out) {
  Pair t{0.0, 0.0};
  for (int k = int(threadIdx.x); k < np; k += 32) {
    pair_add(t, part[k].s);
    t.c += part[k].c;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double s = __shfl_xor_sync(0xffffffffu, t.s, o);
    const double c = __shfl_xor_sync(0xffffffffu, t.c, o);
    pair_add(t, s);
    t.c += c;
  }
  if (threadIdx.x == 0) {
    *slot = t;
    *out = t.s + t.c;
  }
}

std::mutex g_mu;
constexpr int kMaxDevices = 64;
Pair* g_scratch_ptr[kMaxDevices] = {};

int scratch_for_current_device(Pair** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cfdb_cuda_fail(nullptr, e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return cfdb_fail(nullptr, CFDB_EUNSUPPORTED, "device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cfdb_cuda_fail(nullptr, e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_scratch_ptr[dev] = static_cast<Pair*>(p);
  }
  *out = g_scratch_ptr[dev];
  return CFDB_OK;
}

}  // namespace

extern "C" int cfdb_total_fp64_noalloc(int dtype, const void* field, const void* volumes, double volume, int64_t n,
                                       void* stream, double* out_device) {
  if (!dtype_ok(dtype)) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_total_fp64_noalloc: unknown dtype %d", dtype);
  if (!out_device) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_total_fp64_noalloc: out_device is NULL");
  if (n < 0) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_total_fp64_noalloc: negative n");
  if (n > kMaxChunks * kChunk)
    return cfdb_fail(nullptr, CFDB_EINVAL,
                     "cfdb_total_fp64_noalloc: n = %lld exceeds the allocation-free maximum of %lld cells",
                     (long long)n, kMaxChunks * kChunk);
  if (n > 0 && !field) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_total_fp64_noalloc: field is NULL");
  if (!volumes && !std::isfinite(volume))
    return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_total_fp64_noalloc: volume must be finite");
  Pair* scratch = nullptr;
  if (int rc = scratch_for_current_device(&scratch)) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int chunks = int((n + kChunk - 1) / kChunk);
  if (chunks > 0) {
    if (dtype == CFDB_F64)
      chunk_total_k<double><<<chunks, kThreads, 0, s>>>(static_cast<const double*>(field),
                                                         static_cast<const double*>(volumes), volume, n, scratch);
    else
      chunk_total_k<float><<<chunks, kThreads, 0, s>>>(static_cast<const float*>(field),
                                                        static_cast<const float*>(volumes), volume, n, scratch);
  }
  chunk_final_k<<<1, 32, 0, s>>>(scratch, chunks, scratch + kMaxChunks, out_device);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cfdb_cuda_fail(nullptr, e, "cfdb_total_fp64_noalloc launch");
  return CFDB_OK;
}
