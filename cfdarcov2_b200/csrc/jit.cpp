// Run-time compiled kernels: the role of the reference's KernelBuilder
// (src/fvm3d.cpp:1219-1394), which hands a generated CUDA source to OCCA.
// Here NVRTC compiles the source for sm_100a into a cubin, the CUDA runtime
// loads it as a library (cudaLibraryLoadData) and launches the entry point
// on the context's stream.  Modules are cached per context by source text,
// compiled cubins on disk across processes, and a batch of sources compiles
// on several host threads.
//
// Generated sources may include "cfdb_jit.cuh" (kJitHeader below): the
// operator layer's Green-Gauss gradient, orthogonal Laplacian and the two
// stages of the stabilisation as device templates over a callable that
// reads the operand at any cell and over the geometry (face arrays, or the
// constants of an exact lattice).  Their arithmetic and its order are those
// of plain_ops.cu's grad_k, lapl_at and stab1_k/stab2_k; compiled with
// --fmad=false and IEEE division as plain_ops.cu is, a generated kernel
// rounds exactly like the chain of operator kernels it replaces.
#include <nvrtc.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "cfdb_internal.hpp"

namespace {

const char* kJitHeader = R"CFDB(
#pragma once
// Geometry of a generated kernel, read through accessors so that one set of
// operator templates serves both forms: CfdbGeom reads the per-face arrays
// (entry (i, f) at f*n + i, per-dimension arrays stacked at d*6n), and
// CfdbLattice<C> takes the per-slot constants of an exact lattice and derives
// the neighbour ids and wall faces from the cell index.  Both give the same
// values, so the operator arithmetic rounds the same.
struct CfdbGeom {
  const int* ids;
  const float* normal;
  const float* normal_alt;
  const float* area_;
  const float* alpha_;
  const float* len_;
  const float* volume_;
  long long n;
  __device__ __forceinline__ long long count() const { return n; }
  __device__ __forceinline__ long long id(int f, long long i) const { return (long long)ids[f * n + i]; }
  __device__ __forceinline__ float nrm(int d, int f, long long i) const { return normal[d * 6 * n + f * n + i]; }
  __device__ __forceinline__ float nalt(int d, int f, long long i) const { return normal_alt[d * 6 * n + f * n + i]; }
  __device__ __forceinline__ float area(int f, long long i) const { return area_[f * n + i]; }
  __device__ __forceinline__ float alpha(int f, long long i) const { return alpha_[f * n + i]; }
  __device__ __forceinline__ float len(int f, long long i) const { return len_[f * n + i]; }
  __device__ __forceinline__ float volume(long long i) const { return volume_[i]; }
  __device__ __forceinline__ static constexpr bool nrm_nonzero(int, int) { return true; }
  __device__ __forceinline__ static constexpr bool nalt_nonzero(int, int) { return true; }
};

// C: a generated struct with the lattice's dimensions (NX, NY, NZ) and its
// per-slot constants as constexpr functions (nrm(k), nalt(k) with k = d*6 + f;
// area(f); alpha(k), len(k) with k = wall*6 + f; volume()).  Known at
// compile time, a zero normal component drops its face term: the term is
// +-0, and adding +-0 to an accumulator that starts at +0 never changes it,
// so for finite operands the sum keeps the array form's bits.
template <class C> struct CfdbLattice {
  __device__ __forceinline__ static constexpr long long count() { return C::NX * C::NY * C::NZ; }
  __device__ __forceinline__ static bool wall(int f, long long i) {
    long long x, y, z;
    if (count() < (1LL << 31)) {  // 32-bit division by constants
      const unsigned ii = (unsigned)i, pl = (unsigned)(C::NY * C::NZ);
      const unsigned xx = ii / pl, r = ii - xx * pl, yy = r / (unsigned)C::NZ;
      x = xx, y = yy, z = r - yy * (unsigned)C::NZ;
    } else {
      x = i / (C::NY * C::NZ);
      const long long r = i - x * (C::NY * C::NZ);
      y = r / C::NZ, z = r - y * C::NZ;
    }
    switch (f) {
      case 0: return z == 0;
      case 1: return z == C::NZ - 1;
      case 2: return y == 0;
      case 3: return y == C::NY - 1;
      case 4: return x == 0;
      default: return x == C::NX - 1;
    }
  }
  __device__ __forceinline__ static long long id(int f, long long i) {
    const long long step = f == 0 ? -1LL : f == 1 ? 1LL : f == 2 ? -C::NZ : f == 3 ? C::NZ
                         : f == 4 ? -C::NY * C::NZ : C::NY * C::NZ;
    return wall(f, i) ? i : i + step;
  }
  __device__ __forceinline__ static constexpr bool nrm_nonzero(int d, int f) { return C::nrm(d * 6 + f) != 0.f; }
  __device__ __forceinline__ static constexpr bool nalt_nonzero(int d, int f) { return C::nalt(d * 6 + f) != 0.f; }
  __device__ __forceinline__ static float nrm(int d, int f, long long) { return C::nrm(d * 6 + f); }
  __device__ __forceinline__ static float nalt(int d, int f, long long) { return C::nalt(d * 6 + f); }
  __device__ __forceinline__ static float area(int f, long long) { return C::area(f); }
  __device__ __forceinline__ static float alpha(int f, long long i) { return C::alpha((wall(f, i) ? 6 : 0) + f); }
  __device__ __forceinline__ static float len(int f, long long i) { return C::len((wall(f, i) ? 6 : 0) + f); }
  __device__ __forceinline__ static float volume(long long) { return C::volume(); }
};

// Green-Gauss gradient, component mask (bit d: d/dx_d), faces take the mean
// of the two cells (GradVar, src/fvm3d.cpp:768-829)
template <class F, class G> __device__ __forceinline__ float cfdb_grad(F phi, long long i, int mask, const G& g) {
  const float crr = phi(i);
  float nb[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) nb[f] = phi(g.id(f, i));
  float res = 0.f;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    float acc = 0.f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      if (!g.nalt_nonzero(d, f)) continue;
      const float itp = (crr + nb[f]) * 0.5f;
      const float t = itp * g.nalt(d, f, i);
      acc = acc + t * g.area(f, i);
    }
    const float gd = acc / g.volume(i);
    if (mask & (1 << d)) res = res + gd;
  }
  return res;
}

// one gradient component at cell j (StabVar stage 1)
template <class F, class G> __device__ __forceinline__ float cfdb_grad_component(F phi, long long j, int d, const G& g) {
  const float crr = phi(j);
  float acc = 0.f;
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    if (!g.nalt_nonzero(d, f)) continue;
    const float itp = (crr + phi(g.id(f, j))) * 0.5f;
    const float t = itp * g.nalt(d, f, j);
    acc = acc + t * g.area(f, j);
  }
  return acc / g.volume(j);
}

// orthogonal Laplacian, component mask (Grad2Var, src/fvm3d.cpp:831-906)
template <class F, class G> __device__ __forceinline__ float cfdb_lapl(F phi, long long i, int mask, const G& g) {
  const float crr = phi(i);
  float sn[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) sn[f] = (phi(g.id(f, i)) - crr) * g.alpha(f, i);
  float res = 0.f;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (!(mask & (1 << d))) continue;
    float acc = 0.f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      if (!g.nrm_nonzero(d, f)) continue;
      const float t = sn[f] * g.nrm(d, f, i);
      acc = acc + t * g.area(f, i);
    }
    res = res + acc / g.volume(i);
  }
  return res;
}

// two-stage stabilisation (StabVar, src/fvm3d.cpp:909-942).  Stage 1, per
// cell: the upwind face values phi_P + |x_f - x_P| g_d n_alt of its six
// faces in all three directions, into up (3 x 6n, entry d*6n + f*n + i).
template <class F, class G> __device__ __forceinline__ void cfdb_stab1(F phi, long long i, float* up, const G& g) {
  const long long n = g.count();
  const float crr = phi(i);
  float gr[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) gr[d] = cfdb_grad_component(phi, i, d, g);
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int f = 0; f < 6; ++f) up[d * 6 * n + f * n + i] = crr + g.len(f, i) * gr[d] * g.nalt(d, f, i);
}
// Stage 2: half the jump of the two face values across each face, summed
// over the faces (each cell's face f meets its neighbour's face f ^ 1).
template <class G> __device__ __forceinline__ float cfdb_stab2(const float* up, long long i, int mask, const G& g) {
  const long long n = g.count();
  float res = 0.f;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (!(mask & (1 << d))) continue;
    const float* u = up + d * 6 * n;
    float acc = 0.f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const float col = u[(f ^ 1) * n + g.id(f, i)];
      const float s = 0.5f * (u[f * n + i] - col);
      const float t = s * g.nrm(d, f, i);
      acc = acc + t * g.area(f, i);
    }
    res = res + acc / g.volume(i);
  }
  return res;
}

// The same stabilisation with a 3-float stage 1: the gradient components of
// the operand per cell (gr, 3 x n, entry d*n + i); stage 2 rebuilds each face
// value phi_j + |x_f - x_j| g_d(j) n_alt from phi, gr and the geometry with
// the stage-1 formula, so the result has the two-stage form's bits while the
// pass in between stores 12 bytes per cell instead of 72.
template <class F, class G> __device__ __forceinline__ void cfdb_stab_grad(F phi, long long i, float* gr, const G& g) {
  const long long n = g.count();
#pragma unroll
  for (int d = 0; d < 3; ++d) gr[d * n + i] = cfdb_grad_component(phi, i, d, g);
}
template <class F, class G>
__device__ __forceinline__ float cfdb_stab2g(F phi, const float* gr, long long i, int mask, const G& g) {
  const long long n = g.count();
  const float crr = phi(i);
  float res = 0.f;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (!(mask & (1 << d))) continue;
    const float gi = gr[d * n + i];
    float acc = 0.f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      if (!g.nrm_nonzero(d, f)) continue;
      const long long j = g.id(f, i);
      const float own = crr + g.len(f, i) * gi * g.nalt(d, f, i);
      const float col = phi(j) + g.len(f ^ 1, j) * gr[d * n + j] * g.nalt(d, f ^ 1, j);
      const float s = 0.5f * (own - col);
      const float t = s * g.nrm(d, f, i);
      acc = acc + t * g.area(f, i);
    }
    res = res + acc / g.volume(i);
  }
  return res;
}
)CFDB";

struct Module {
  cudaLibrary_t lib = nullptr;
  std::string log;
};

// modules of every context, by context and source text (a context owns its
// modules until it is destroyed); contexts may live on different host
// threads, so the table is guarded by modules_mutex()
std::map<const cfdb_ctx*, std::map<std::string, std::shared_ptr<Module>>>& modules() {
  static std::map<const cfdb_ctx*, std::map<std::string, std::shared_ptr<Module>>> m;
  return m;
}
std::mutex& modules_mutex() {
  static std::mutex mu;
  return mu;
}

const char* const kOpts[] = {"--gpu-architecture=sm_100a", "--fmad=false", "--prec-div=true", "--prec-sqrt=true",
                             "--ftz=false", "-std=c++17"};

// One NVRTC compile of source into a cubin (thread-safe: touches no context).
struct Compiled {
  std::vector<char> cubin;
  std::string log;
  std::string error;  // empty on success
  bool compile_error = false;
};

Compiled compile_cubin(const std::string& source) {
  Compiled c;
  nvrtcProgram prog = nullptr;
  const char* headers[] = {kJitHeader};
  const char* names[] = {"cfdb_jit.cuh"};
  nvrtcResult r = nvrtcCreateProgram(&prog, source.c_str(), "cfdb_generated.cu", 1, headers, names);
  if (r != NVRTC_SUCCESS) {
    c.error = std::string("nvrtcCreateProgram: ") + nvrtcGetErrorString(r);
    return c;
  }
  r = nvrtcCompileProgram(prog, int(sizeof(kOpts) / sizeof(kOpts[0])), kOpts);
  size_t log_size = 0;
  nvrtcGetProgramLogSize(prog, &log_size);
  c.log.assign(log_size, '\0');
  if (log_size > 1) nvrtcGetProgramLog(prog, &c.log[0]);
  if (r != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    c.compile_error = true;
    c.error = std::string("generated kernel does not compile: ") + nvrtcGetErrorString(r) + "\n" + c.log;
    return c;
  }
  size_t cubin_size = 0;
  r = nvrtcGetCUBINSize(prog, &cubin_size);
  c.cubin.resize(cubin_size);
  if (r == NVRTC_SUCCESS) r = nvrtcGetCUBIN(prog, c.cubin.data());
  nvrtcDestroyProgram(&prog);
  if (r != NVRTC_SUCCESS) c.error = std::string("nvrtcGetCUBIN: ") + nvrtcGetErrorString(r);
  return c;
}

// ---- on-disk cache of compiled kernels --------------------------------------
// The role of OCCA's kernel cache behind the reference's KernelBuilder: a
// generated source compiled once is loaded from disk by later processes.
// Directory: $CFDB_KERNEL_CACHE, else $XDG_CACHE_HOME/cfdb_kernels, else
// $HOME/.cache/cfdb_kernels; CFDB_KERNEL_CACHE=off disables it.  An entry is
// <hash>.cubin holding a magic word, the key text (compiler version, options,
// header and source) and the cubin; a key that differs in any byte misses.
// Unwritable directories and damaged entries fall back to compiling.
std::string cache_dir() {
  const char* e = std::getenv("CFDB_KERNEL_CACHE");
  if (e && std::strcmp(e, "off") == 0) return std::string();
  if (e && *e) return e;
  const char* x = std::getenv("XDG_CACHE_HOME");
  if (x && *x) return std::string(x) + "/cfdb_kernels";
  const char* h = std::getenv("HOME");
  if (h && *h) return std::string(h) + "/.cache/cfdb_kernels";
  return std::string();
}

std::string cache_key(const std::string& source) {
  int major = 0, minor = 0;
  nvrtcVersion(&major, &minor);
  std::string k = "nvrtc " + std::to_string(major) + "." + std::to_string(minor) + "\n";
  for (const char* o : kOpts) k += std::string(o) + "\n";
  k += kJitHeader;
  k += "\n--\n";
  k += source;
  return k;
}

uint64_t fnv1a(const std::string& s) {
  uint64_t h = 1469598103934665603ull;
  for (unsigned char ch : s) {
    h ^= ch;
    h *= 1099511628211ull;
  }
  return h;
}

std::string cache_path(const std::string& dir, const std::string& key) {
  char name[32];
  std::snprintf(name, sizeof(name), "/%016llx.cubin", (unsigned long long)fnv1a(key));
  return dir + name;
}

constexpr uint64_t kCacheMagic = 0x31424e4942424443ull;  // "CDBBINB1"

bool cache_load(const std::string& key, std::vector<char>& cubin) {
  const std::string dir = cache_dir();
  if (dir.empty()) return false;
  FILE* f = std::fopen(cache_path(dir, key).c_str(), "rb");
  if (!f) return false;
  bool ok = false;
  uint64_t magic = 0, klen = 0, blen = 0;
  if (std::fread(&magic, 8, 1, f) == 1 && magic == kCacheMagic && std::fread(&klen, 8, 1, f) == 1 &&
      klen == key.size()) {
    std::string k(klen, '\0');
    if (std::fread(&k[0], 1, klen, f) == klen && k == key && std::fread(&blen, 8, 1, f) == 1 && blen > 0 &&
        blen < (1ull << 30)) {
      cubin.resize(blen);
      ok = std::fread(cubin.data(), 1, blen, f) == blen;
    }
  }
  std::fclose(f);
  return ok;
}

void cache_store(const std::string& key, const std::vector<char>& cubin) {
  const std::string dir = cache_dir();
  if (dir.empty()) return;
  std::error_code ec;
  std::filesystem::create_directories(dir, ec);
  const std::string path = cache_path(dir, key);
  const std::string tmp = path + ".tmp" + std::to_string(long(getpid())) + "_" +
                          std::to_string(uint64_t(std::hash<std::thread::id>{}(std::this_thread::get_id())));
  FILE* f = std::fopen(tmp.c_str(), "wb");
  if (!f) return;
  const uint64_t klen = key.size(), blen = cubin.size();
  bool ok = std::fwrite(&kCacheMagic, 8, 1, f) == 1 && std::fwrite(&klen, 8, 1, f) == 1 &&
            std::fwrite(key.data(), 1, klen, f) == klen && std::fwrite(&blen, 8, 1, f) == 1 &&
            std::fwrite(cubin.data(), 1, blen, f) == blen;
  ok = std::fclose(f) == 0 && ok;
  if (ok) std::filesystem::rename(tmp, path, ec);
  if (!ok || ec) std::filesystem::remove(tmp, ec);
}

}  // namespace

struct cfdb_kernel {
  cfdb_ctx* ctx = nullptr;
  std::shared_ptr<Module> mod;
  cudaKernel_t kern = nullptr;
};

// Releases the modules of a context (called when it is destroyed).
void cfdb_jit_release(cfdb_ctx* ctx) {
  std::lock_guard<std::mutex> lock(modules_mutex());
  auto it = modules().find(ctx);
  if (it == modules().end()) return;
  for (auto& kv : it->second)
    if (kv.second->lib) cudaLibraryUnload(kv.second->lib);
  modules().erase(it);
}

extern "C" int cfdb_kernel_build_many(cfdb_ctx* ctx, int count, const char* const* sources, const char* const* names,
                                      cfdb_kernel** out) {
  CfdbRange range_("cfdb_kernel_build_many");
  if (!out || count < 0 || (count > 0 && (!sources || !names)))
    return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_kernel_build_many: bad arguments");
  for (int k = 0; k < count; ++k) out[k] = nullptr;
  if (!ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_kernel_build_many: ctx is NULL");
  for (int k = 0; k < count; ++k)
    if (!sources[k] || !names[k] || !*names[k]) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_kernel_build: NULL argument");
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  std::lock_guard<std::mutex> lock(modules_mutex());  // held through the build: one context's table at a time
  auto& mine = modules()[ctx];
  // distinct sources without a module in this context: from the disk cache or compiled, in parallel
  std::vector<std::string> todo;
  for (int k = 0; k < count; ++k)
    if (!mine.count(sources[k]) && std::find(todo.begin(), todo.end(), sources[k]) == todo.end())
      todo.emplace_back(sources[k]);
  std::vector<Compiled> built(todo.size());
  std::atomic<size_t> next{0};
  auto worker = [&] {
    for (size_t j; (j = next.fetch_add(1)) < todo.size();) {
      const std::string key = cache_key(todo[j]);
      if (cache_load(key, built[j].cubin)) continue;
      built[j] = compile_cubin(todo[j]);
      if (built[j].error.empty()) cache_store(key, built[j].cubin);
    }
  };
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nthreads = std::min(todo.size(), std::min<size_t>(hw, 32));
  std::vector<std::thread> pool;
  for (size_t t = 1; t < nthreads; ++t) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
  for (size_t j = 0; j < todo.size(); ++j) {
    if (!built[j].error.empty())
      return cfdb_fail(ctx, built[j].compile_error ? CFDB_EINVAL : CFDB_ECUDA, "%s", built[j].error.c_str());
    auto mod = std::make_shared<Module>();
    mod->log = built[j].log;
    CFDB_CUDA(ctx, cudaLibraryLoadData(&mod->lib, built[j].cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
    mine[todo[j]] = mod;
  }
  for (int k = 0; k < count; ++k) {
    auto kp = std::make_unique<cfdb_kernel>();
    kp->ctx = ctx;
    kp->mod = mine[sources[k]];
    cudaError_t e = cudaLibraryGetKernel(&kp->kern, kp->mod->lib, names[k]);
    if (e != cudaSuccess) {
      cudaGetLastError();
      for (int j = 0; j < k; ++j) {
        cfdb_kernel_destroy(out[j]);
        out[j] = nullptr;
      }
      return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_kernel_build: no extern \"C\" __global__ %s in the source", names[k]);
    }
    cfdb_kernel* raw = kp.release();
    cfdb_adopt(ctx, raw, [raw] { raw->ctx = nullptr; });  // the module dies with the context
    out[k] = raw;
  }
  return CFDB_OK;
}

extern "C" int cfdb_kernel_build(cfdb_ctx* ctx, const char* source, const char* name, cfdb_kernel** out) {
  if (!out) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_kernel_build: out is NULL");
  return cfdb_kernel_build_many(ctx, 1, &source, &name, out);
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

extern "C" int cfdb_kernel_info(const cfdb_kernel* k, int* registers, int64_t* local_bytes, int* max_threads) {
  if (!k || !k->ctx) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_kernel_info: kernel is NULL or its context was destroyed");
  cudaFuncAttributes fa{};
  CFDB_CUDA(k->ctx, cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(k->kern)));
  if (registers) *registers = fa.numRegs;
  if (local_bytes) *local_bytes = int64_t(fa.localSizeBytes);
  if (max_threads) *max_threads = fa.maxThreadsPerBlock;
  return CFDB_OK;
}

extern "C" int cfdb_kernel_destroy(cfdb_kernel* k) {
  if (!k) return CFDB_OK;
  if (k->ctx) cfdb_release(k->ctx, k);
  delete k;  // the module stays cached with its context
  return CFDB_OK;
}
