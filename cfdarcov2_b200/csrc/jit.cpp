// Run-time compiled kernels: the role of the reference's KernelBuilder
// (src/fvm3d.cpp:1219-1394), which hands a generated CUDA source to OCCA.
// Here NVRTC compiles the source for sm_100a into a cubin, the CUDA runtime
// loads it as a library (cudaLibraryLoadData) and launches the entry point
// on the context's stream.  Modules are cached per context by source text.
//
// Generated sources may include "cfdb_jit.cuh" (kJitHeader below): the
// operator layer's Green-Gauss gradient, orthogonal Laplacian and the two
// stages of the stabilisation as device templates over a callable that
// reads the operand at any cell.  Their arithmetic and its order are those
// of plain_ops.cu's grad_k, lapl_at and stab1_k/stab2_k; compiled with
// --fmad=false and IEEE division as plain_ops.cu is, a generated kernel
// rounds exactly like the chain of operator kernels it replaces.
#include <nvrtc.h>

#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "cfdb_internal.hpp"

namespace {

const char* kJitHeader = R"CFDB(
#pragma once
struct CfdbGeom {
  const int* ids;
  const float* normal;
  const float* normal_alt;
  const float* area;
  const float* alpha;
  const float* len;
  const float* volume;
  long long n;
};

// Green-Gauss gradient, component mask (bit d: d/dx_d), faces take the mean
// of the two cells (GradVar, src/fvm3d.cpp:768-829)
template <class F> __device__ __forceinline__ float cfdb_grad(F phi, long long i, int mask, const CfdbGeom& g) {
  const long long n = g.n;
  const float crr = phi(i);
  float nb[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) nb[f] = phi((long long)g.ids[f * n + i]);
  float res = 0.f;
  for (int d = 0; d < 3; ++d) {
    float acc = 0.f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const long long k6 = f * n + i;
      const float itp = (crr + nb[f]) * 0.5f;
      const float t = itp * g.normal_alt[d * 6 * n + k6];
      acc = acc + t * g.area[k6];
    }
    const float gd = acc / g.volume[i];
    if (mask & (1 << d)) res = res + gd;
  }
  return res;
}

// one gradient component at cell j (StabVar stage 1)
template <class F> __device__ __forceinline__ float cfdb_grad_component(F phi, long long j, int d, const CfdbGeom& g) {
  const long long n = g.n;
  const float crr = phi(j);
  float acc = 0.f;
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const long long k6 = f * n + j;
    const float itp = (crr + phi((long long)g.ids[k6])) * 0.5f;
    const float t = itp * g.normal_alt[d * 6 * n + k6];
    acc = acc + t * g.area[k6];
  }
  return acc / g.volume[j];
}

// orthogonal Laplacian, component mask (Grad2Var, src/fvm3d.cpp:831-906)
template <class F> __device__ __forceinline__ float cfdb_lapl(F phi, long long i, int mask, const CfdbGeom& g) {
  const long long n = g.n;
  const float crr = phi(i);
  float sn[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const long long k6 = f * n + i;
    sn[f] = (phi((long long)g.ids[k6]) - crr) * g.alpha[k6];
  }
  float res = 0.f;
  for (int d = 0; d < 3; ++d) {
    if (!(mask & (1 << d))) continue;
    float acc = 0.f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const long long k6 = f * n + i;
      const float t = sn[f] * g.normal[d * 6 * n + k6];
      acc = acc + t * g.area[k6];
    }
    res = res + acc / g.volume[i];
  }
  return res;
}

// two-stage stabilisation (StabVar, src/fvm3d.cpp:909-942).  Stage 1, per
// cell: the upwind face values phi_P + |x_f - x_P| g_d n_alt of its six
// faces in all three directions, into up (3 x 6n, entry d*6n + f*n + i).
template <class F> __device__ __forceinline__ void cfdb_stab1(F phi, long long i, float* up, const CfdbGeom& g) {
  const long long n = g.n;
  const float crr = phi(i);
  float gr[3];
  for (int d = 0; d < 3; ++d) gr[d] = cfdb_grad_component(phi, i, d, g);
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const long long k6 = f * n + i;
      const long long kd = d * 6 * n + k6;
      up[kd] = crr + g.len[k6] * gr[d] * g.normal_alt[kd];
    }
}
// Stage 2: half the jump of the two face values across each face, summed
// over the faces (each cell's face f meets its neighbour's face f ^ 1).
__device__ __forceinline__ float cfdb_stab2(const float* up, long long i, int mask, const CfdbGeom& g) {
  const long long n = g.n;
  float res = 0.f;
  for (int d = 0; d < 3; ++d) {
    if (!(mask & (1 << d))) continue;
    const float* u = up + d * 6 * n;
    float acc = 0.f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const long long k6 = f * n + i;
      const float col = u[(f ^ 1) * n + g.ids[k6]];
      const float s = 0.5f * (u[k6] - col);
      const float t = s * g.normal[d * 6 * n + k6];
      acc = acc + t * g.area[k6];
    }
    res = res + acc / g.volume[i];
  }
  return res;
}
)CFDB";

struct Module {
  cudaLibrary_t lib = nullptr;
  std::string log;
};

// modules of every context, by context and source text (a context owns its
// modules until it is destroyed)
std::map<const cfdb_ctx*, std::map<std::string, std::shared_ptr<Module>>>& modules() {
  static std::map<const cfdb_ctx*, std::map<std::string, std::shared_ptr<Module>>> m;
  return m;
}

int compile(cfdb_ctx* ctx, const std::string& source, std::shared_ptr<Module>& out) {
  nvrtcProgram prog = nullptr;
  const char* headers[] = {kJitHeader};
  const char* names[] = {"cfdb_jit.cuh"};
  nvrtcResult r = nvrtcCreateProgram(&prog, source.c_str(), "cfdb_generated.cu", 1, headers, names);
  if (r != NVRTC_SUCCESS) return cfdb_fail(ctx, CFDB_ECUDA, "nvrtcCreateProgram: %s", nvrtcGetErrorString(r));
  const char* opts[] = {"--gpu-architecture=sm_100a", "--fmad=false", "--prec-div=true", "--prec-sqrt=true",
                        "--ftz=false", "-std=c++17"};
  r = nvrtcCompileProgram(prog, int(sizeof(opts) / sizeof(opts[0])), opts);
  size_t log_size = 0;
  nvrtcGetProgramLogSize(prog, &log_size);
  std::string log(log_size, '\0');
  if (log_size > 1) nvrtcGetProgramLog(prog, &log[0]);
  if (r != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    return cfdb_fail(ctx, CFDB_EINVAL, "generated kernel does not compile: %s\n%s", nvrtcGetErrorString(r), log.c_str());
  }
  size_t cubin_size = 0;
  r = nvrtcGetCUBINSize(prog, &cubin_size);
  std::vector<char> cubin(cubin_size);
  if (r == NVRTC_SUCCESS) r = nvrtcGetCUBIN(prog, cubin.data());
  nvrtcDestroyProgram(&prog);
  if (r != NVRTC_SUCCESS) return cfdb_fail(ctx, CFDB_ECUDA, "nvrtcGetCUBIN: %s", nvrtcGetErrorString(r));
  auto mod = std::make_shared<Module>();
  mod->log = log;
  CFDB_CUDA(ctx, cudaLibraryLoadData(&mod->lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
  out = std::move(mod);
  return CFDB_OK;
}

}  // namespace

struct cfdb_kernel {
  cfdb_ctx* ctx = nullptr;
  std::shared_ptr<Module> mod;
  cudaKernel_t kern = nullptr;
};

// Releases the modules of a context (called when it is destroyed).
void cfdb_jit_release(cfdb_ctx* ctx) {
  auto it = modules().find(ctx);
  if (it == modules().end()) return;
  for (auto& kv : it->second)
    if (kv.second->lib) cudaLibraryUnload(kv.second->lib);
  modules().erase(it);
}

extern "C" int cfdb_kernel_build(cfdb_ctx* ctx, const char* source, const char* name, cfdb_kernel** out) {
  if (!out) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_kernel_build: out is NULL");
  *out = nullptr;
  if (!ctx || !source || !name || !*name) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_kernel_build: NULL argument");
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  auto& mine = modules()[ctx];
  std::shared_ptr<Module> mod;
  auto hit = mine.find(source);
  if (hit != mine.end()) {
    mod = hit->second;
  } else {
    if (int rc = compile(ctx, source, mod)) return rc;
    mine[source] = mod;
  }
  auto k = std::make_unique<cfdb_kernel>();
  k->ctx = ctx;
  k->mod = mod;
  cudaError_t e = cudaLibraryGetKernel(&k->kern, mod->lib, name);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_kernel_build: no extern \"C\" __global__ %s in the source", name);
  }
  cfdb_kernel* kp = k.release();
  cfdb_adopt(ctx, kp, [kp] { kp->ctx = nullptr; });  // the module dies with the context
  *out = kp;
  return CFDB_OK;
}

extern "C" int cfdb_kernel_launch(cfdb_kernel* k, int64_t n_threads, int block, void** args) {
  if (!k || !k->ctx)
    return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_kernel_launch: kernel is NULL or its context was destroyed");
  cfdb_ctx* ctx = k->ctx;
  if (n_threads < 0 || block < 32 || block > 1024 || block % 32)
    return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_kernel_launch: bad launch shape");
  if (n_threads == 0) return CFDB_OK;
  const int64_t blocks = (n_threads + block - 1) / block;
  if (blocks > 2147483647LL) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_kernel_launch: too many threads");
  CFDB_CUDA(ctx, cudaLaunchKernel(reinterpret_cast<const void*>(k->kern), dim3(unsigned(blocks)), dim3(unsigned(block)),
                                  args, 0, ctx->stream));
  CFDB_LAUNCHED(ctx);
  return CFDB_OK;
}

extern "C" int cfdb_kernel_destroy(cfdb_kernel* k) {
  if (!k) return CFDB_OK;
  if (k->ctx) cfdb_release(k->ctx, k);
  delete k;  // the module stays cached with its context
  return CFDB_OK;
}
