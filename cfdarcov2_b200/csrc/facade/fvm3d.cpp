// Implementation of the drop-in C++ facade (include/cfdb/*.hpp).  It only
// uses libcfdb's C ABI: every field lives in library device buffers and every
// expression node evaluates through a cfdb_op_* kernel into a buffer it
// allocates once.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <filesystem>
#include <map>
#include <set>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <unordered_map>
#include <utility>

#include "cfdb/fvm3d.hpp"

namespace cfdb {

void check(int status, const char* what) {
  if (status != CFDB_OK) {
    std::string msg = std::string(what) + ": " + cfdb_last_error(CFDArcoGlobalInit::ctx());
    throw std::runtime_error(msg);
  }
}

// ---------------------------------------------------------------------------
// global context
// ---------------------------------------------------------------------------
namespace {
cfdb_ctx* g_ctx = nullptr;
}

bool CFDArcoGlobalInit::skip_history = true;
bool CFDArcoGlobalInit::cuda_enabled = false;
bool CFDArcoGlobalInit::store_stepping = false;
bool CFDArcoGlobalInit::jit_lattice = true;
bool CFDArcoGlobalInit::jit_all = true;
bool CFDArcoGlobalInit::jit_report = false;
std::string CFDArcoGlobalInit::store_dir;

void CFDArcoGlobalInit::initialize(int, char**, bool skip_hist, const std::string& store_path) {
  skip_history = skip_hist;
  const std::time_t t = std::time(nullptr);
  const std::tm* now = std::localtime(&t);
  char stamp[96];
  std::snprintf(stamp, sizeof(stamp), "run_%d_%d_%d_%d_%d_%d", now->tm_year + 1900, now->tm_mon + 1, now->tm_mday,
                now->tm_hour, now->tm_min, now->tm_sec);
  store_dir = (std::filesystem::path(store_path) / stamp).string();
}

void CFDArcoGlobalInit::enable_cuda(int device) {
  if (g_ctx) return;
  cfdb_ctx* c = nullptr;
  if (cfdb_ctx_create(device, &c) != CFDB_OK)
    throw std::runtime_error(std::string("cfdb_ctx_create: ") + cfdb_last_error(nullptr));
  g_ctx = c;
  cuda_enabled = true;
}

namespace {
// Device buffers of the facade: freed ones are kept by size and handed out
// again instead of going back to the driver (cudaMalloc of a 100 MB buffer
// costs ~0.7 ms, cudaFree ~0.35 ms), as the reference allocates from an RMM
// pool it reserves at start-up (src/cfdarcho_main_3d.cpp:333-344).  All
// facade work runs on the context's one stream, so a reused buffer is only
// touched after the work that used it before.  The kept buffers go back to
// the device in finalize() and when an allocation fails.
struct BlockCache {
  std::mutex mu;
  std::unordered_map<float*, size_t> live;  // buffer -> floats
  std::multimap<size_t, float*> kept;       // floats -> freed buffer
};
BlockCache& blocks() {
  static BlockCache c;
  return c;
}
void release_kept(cfdb_ctx* ctx) {  // with the cache's lock held
  for (auto& kv : blocks().kept) cfdb_free(ctx, kv.second);
  blocks().kept.clear();
}

float* device_alloc(size_t n) {
  cfdb_ctx* ctx = CFDArcoGlobalInit::ctx();
  BlockCache& c = blocks();
  std::lock_guard<std::mutex> lock(c.mu);
  auto it = c.kept.find(n);
  if (it != c.kept.end()) {
    float* p = it->second;
    c.kept.erase(it);
    c.live[p] = n;
    return p;
  }
  void* p = nullptr;
  int rc = cfdb_alloc(ctx, int64_t(n * sizeof(float)), &p);
  if (rc == CFDB_ENOMEM && !c.kept.empty()) {
    release_kept(ctx);
    rc = cfdb_alloc(ctx, int64_t(n * sizeof(float)), &p);
  }
  check(rc, "cfdb_alloc");
  c.live[static_cast<float*>(p)] = n;
  return static_cast<float*>(p);
}
void device_free(float* p) {
  if (!p || !CFDArcoGlobalInit::cuda_enabled) return;
  BlockCache& c = blocks();
  std::lock_guard<std::mutex> lock(c.mu);
  auto it = c.live.find(p);
  if (it == c.live.end()) {
    cfdb_free(CFDArcoGlobalInit::ctx(), p);
    return;
  }
  c.kept.emplace(it->second, p);
  c.live.erase(it);
}
}  // namespace

void CFDArcoGlobalInit::finalize() {
  if (g_ctx) {
    std::lock_guard<std::mutex> lock(blocks().mu);
    release_kept(g_ctx);
    blocks().live.clear();  // the context frees what is still live
    cfdb_ctx_destroy(g_ctx);
  }
  g_ctx = nullptr;
  cuda_enabled = false;
}

cfdb_ctx* CFDArcoGlobalInit::ctx() {
  if (!g_ctx) enable_cuda(0);
  return g_ctx;
}

// ---------------------------------------------------------------------------
// Mesh3D
// ---------------------------------------------------------------------------
Mesh3D::Mesh3D(size_t x, size_t y, size_t z, float dx, float dy, float dz)
    : _num_nodes(x * y * z), _x(x), _y(y), _z(z), _lx(dx * float(x)), _ly(dy * float(y)), _lz(dz * float(z)),
      _dx(dx), _dy(dy), _dz(dz) {}

Mesh3D::~Mesh3D() {
  if (mesh_ && CFDArcoGlobalInit::cuda_enabled) cfdb_mesh_destroy(mesh_);
}

void Mesh3D::init_basic_internals() {}

void Mesh3D::compute() {
  cfdb_lattice_geometry lat{};
  check(cfdb_mesh_lattice_geometry(handle(), &lat), "cfdb_mesh_lattice_geometry");  // cached in the mesh
}

cfdb_mesh* Mesh3D::handle() {
  if (!mesh_)
    check(cfdb_mesh_create_structured(CFDArcoGlobalInit::ctx(), int64_t(_x), int64_t(_y), int64_t(_z), _dx, _dy,
                                      _dz, &mesh_),
          "cfdb_mesh_create_structured");
  return mesh_;
}

float Mesh3D::x(size_t id) const { return (float(id / (_y * _z)) + 0.5f) * _dx; }
float Mesh3D::y(size_t id) const { return (float((id / _z) % _y) + 0.5f) * _dy; }
float Mesh3D::z(size_t id) const { return (float(id % _z) + 0.5f) * _dz; }
bool Mesh3D::is_boundary(size_t id) const {
  const size_t xi = id / (_y * _z), yi = (id / _z) % _y, zi = id % _z;
  return xi == 0 || yi == 0 || zi == 0 || xi + 1 == _x || yi + 1 == _y || zi + 1 == _z;
}

// ---------------------------------------------------------------------------
// expression nodes
// ---------------------------------------------------------------------------
struct Node {
  enum Kind { kField, kConst, kBinary, kNeg, kGrad, kLapl, kStab, kDt } kind = kConst;
  int op = 0;
  int mask = 7;
  float value = 0.f;
  std::shared_ptr<Node> a, b;
  Variable* field = nullptr;
  const DT* dt = nullptr;
  Mesh3D* mesh = nullptr;
  float* buf = nullptr;
  bool filled = false;
  ~Node() { device_free(buf); }
};

namespace {

std::shared_ptr<Node> make(Node::Kind k, Mesh3D* mesh) {
  auto n = std::make_shared<Node>();
  n->kind = k;
  n->mesh = mesh;
  return n;
}

Mesh3D* mesh_of(const Variable& a, const Variable& b) { return a.mesh ? a.mesh : b.mesh; }

Variable wrap(std::shared_ptr<Node> n) {
  Variable v;
  v.mesh = n->mesh;
  v.node = std::move(n);
  return v;
}

Variable binary(const Variable& l, const Variable& r, int op) {
  auto n = make(Node::kBinary, mesh_of(l, r));
  n->op = op;
  n->a = l.node;
  n->b = r.node;
  return wrap(n);
}

Variable mesh_op(const Variable& v, Node::Kind k, int mask) {
  auto n = make(k, v.mesh);
  n->mask = mask;
  n->a = v.node;
  return wrap(n);
}

const float* eval_node(Node* n) {
  cfdb_ctx* ctx = CFDArcoGlobalInit::ctx();
  const int64_t N = int64_t(n->mesh->_num_nodes);
  if (n->kind == Node::kField) return n->field->current_cu;
  if (!n->buf) n->buf = device_alloc(size_t(N));
  switch (n->kind) {
    case Node::kConst:
      if (!n->filled) {
        check(cfdb_op_fill(ctx, CFDB_F32, n->buf, n->value, N), "cfdb_op_fill");
        n->filled = true;
      }
      break;
    case Node::kDt:
      check(cfdb_op_fill(ctx, CFDB_F32, n->buf, n->dt->_dt, N), "cfdb_op_fill");
      break;
    case Node::kBinary: {
      // a constant operand becomes a scalar operation (no second stream)
      if (n->b->kind == Node::kConst || n->b->kind == Node::kDt) {
        const float s = n->b->kind == Node::kConst ? n->b->value : n->b->dt->_dt;
        check(cfdb_op_scalar(ctx, CFDB_F32, n->op, eval_node(n->a.get()), s, n->buf, N), "cfdb_op_scalar");
      } else if (n->a->kind == Node::kConst || n->a->kind == Node::kDt) {
        const float s = n->a->kind == Node::kConst ? n->a->value : n->a->dt->_dt;
        const int op = n->op == CFDB_OP_SUB ? CFDB_OP_RSUB : (n->op == CFDB_OP_DIV ? CFDB_OP_RDIV : n->op);
        check(cfdb_op_scalar(ctx, CFDB_F32, op, eval_node(n->b.get()), s, n->buf, N), "cfdb_op_scalar");
      } else {
        const float* a = eval_node(n->a.get());
        const float* b = eval_node(n->b.get());
        check(cfdb_op_binary(ctx, CFDB_F32, n->op, a, b, n->buf, N), "cfdb_op_binary");
      }
      break;
    }
    case Node::kNeg:
      check(cfdb_op_neg(ctx, CFDB_F32, eval_node(n->a.get()), n->buf, N), "cfdb_op_neg");
      break;
    case Node::kGrad:
      check(cfdb_op_grad(ctx, n->mesh->handle(), CFDB_F32, eval_node(n->a.get()), n->buf, n->mask), "cfdb_op_grad");
      break;
    case Node::kLapl:
      check(cfdb_op_lapl(ctx, n->mesh->handle(), CFDB_F32, eval_node(n->a.get()), n->buf, n->mask), "cfdb_op_lapl");
      break;
    case Node::kStab:
      check(cfdb_op_stab(ctx, n->mesh->handle(), CFDB_F32, eval_node(n->a.get()), n->buf, n->mask), "cfdb_op_stab");
      break;
    default:
      break;
  }
  return n->buf;
}

// ---- run-time generated equation kernels (KernelBuilder, src/fvm3d.cpp:1071-1394)
// An equation becomes a short plan of generated kernels: the pointwise part
// of the right-hand side, the operators and the time update fuse into the
// last one.  An operator whose operand is a pointwise expression of fields
// evaluates it at the neighbours inline; an operand that holds operators
// itself is first materialised in a pass of its own (so no cell recomputes a
// neighbour's neighbour operators), and a stabilisation first stores the
// operand's gradient (3 floats per cell) in a pass of its own.  Inside a
// kernel there is one device function per expression node, e<k>(i, A) = the
// node's value at cell i.
// Operand order and constants are those of the operator path (a constant
// operand as a scalar operation), and the library compiles with
// --fmad=false, so the plan's result equals the operator chain's bit for
// bit.

// Cells per thread of the generated kernels (JitPlan::cells).
// Measured on the reference's benchmark systems: the single-equation wave
// kernel 206 -> 308 G cell-updates/s at 4 cells per thread (400^3; 8 cells
// per thread fall back to 239 G); the
// Euler system's group kernels lose with 2 (7.4 -> 6.6 G at 200^3: the
// 9-member group's registers double) and its stab passes are level.
// Cell indices stay 64-bit: 32-bit indices (an int index type in the
// operator header for meshes below 2^31 / 18 cells) cut the largest group's
// registers from 80 to 72 but slowed the Euler system from 214 to 229 ms per
// 200 steps at 200^3; __launch_bounds__(256, 4) on the group kernels (64
// registers, 40 bytes of spills in the largest) ran 220 ms; CTAs tiled as
// 32 z x 8 y cells of cpt consecutive x planes (y neighbours from the same
// CTA, x neighbours from the thread's own cells) ran 236 ms against 206 ms
// for the linear chunks.
constexpr int kCptEquation = 4;
constexpr int kCptGroup = 1;
constexpr int kCptStab = 1;

// An input of a generated kernel: a field's current buffer (looked up at
// launch time: fields swap buffers every step) or a scratch buffer of the plan.
struct JitInput {
  Variable* field = nullptr;
  int scratch = -1;
  bool operator==(const JitInput& o) const { return field == o.field && scratch == o.scratch; }
};

struct JitPass {
  cfdb_kernel* k = nullptr;
  std::string source, entry;  // compiled by jit_compile, all passes of all equations at once
  std::vector<JitInput> inputs;
  int out_scratch = -1;  // -1: the equation's output (the last pass)
  // a multi-output pass (a group, the merged stab stage 1): signature (A, n),
  // A.o[k] = outputs[k]: a field's next buffer or a scratch buffer
  bool multi = false;
  std::vector<JitInput> outputs;
  int cpt = 1;  // cells per thread (consecutive chunks of the CTA size)
  ~JitPass() {
    if (k) cfdb_kernel_destroy(k);
  }
};

struct JitPlan {
  Mesh3D* mesh = nullptr;
  // an exact lattice: the kernels take per-slot geometry constants instead of the face arrays
  bool lattice = false;
  cfdb_lattice_geometry lat{};
  std::string geom_type() const { return lattice ? "CfdbLattice<CfdbC>" : "CfdbGeom"; }
  // Kernel body over `cpt` cells per thread, i = chunk start + c x CTA size:
  // every cell's values are computed (`compute`, may use c and i) before any
  // is stored (`store`), so the loads of all of a thread's cells are in
  // flight together: a one-cell thread has two DRAM misses in flight (its
  // new plane and its previous value), too few to cover the DRAM latency.
  static std::string cells(int cpt, const std::string& decls, const std::string& compute, const std::string& store) {
    const std::string c = std::to_string(cpt);
    return "  const long long i0 = (long long)blockIdx.x * (blockDim.x * " + c + ") + threadIdx.x;\n" + decls +
           "#pragma unroll\n  for (int c = 0; c < " + c + "; ++c) {\n"
           "    const long long i = i0 + (long long)c * blockDim.x;\n    if (i < n) {\n" + compute + "    }\n  }\n"
           "#pragma unroll\n  for (int c = 0; c < " + c + "; ++c) {\n"
           "    const long long i = i0 + (long long)c * blockDim.x;\n    if (i < n) {\n" + store + "    }\n  }\n";
  }
  // the lattice's dimensions and constants as compile-time values of the source
  std::string lattice_struct() const {
    if (!lattice) return std::string();
    auto hex = [](float v) {
      char b[40];
      std::snprintf(b, sizeof(b), "%af", double(v));
      return std::string(b);
    };
    auto fn = [&](const char* name, const float* v, int count) {
      std::string f = "  __device__ static constexpr float " + std::string(name) + "(int k) {\n    switch (k) {\n";
      for (int k = 0; k < count; ++k) f += "      case " + std::to_string(k) + ": return " + hex(v[k]) + ";\n";
      return f + "      default: return 0.f;\n    }\n  }\n";
    };
    std::string s = "struct CfdbC {\n  static constexpr long long NX = " + std::to_string(lat.nx) +
                    "LL, NY = " + std::to_string(lat.ny) + "LL, NZ = " + std::to_string(lat.nz) + "LL;\n";
    s += fn("nrm", lat.normal, 18) + fn("nalt", lat.normal_alt, 18) + fn("area", lat.area, 6) +
         fn("alpha", lat.alpha, 12) + fn("len", lat.len, 12);
    s += "  __device__ static constexpr float volume() { return " + hex(lat.volume) + "; }\n};\n";
    return s;
  }
  std::vector<std::unique_ptr<JitPass>> passes;  // run order; the last computes the equation
  // scratch buffers: sizes while planning; placed in one block that the
  // caller allocates for all plans of a system (place_scratch)
  std::vector<size_t> scratch_floats;
  std::vector<float*> scratch;
  std::map<const Node*, int> materialised;
  std::map<const void*, int> stab_grads;  // by field, or by operand node
  bool ok = true;
  int new_scratch(size_t floats) {
    scratch_floats.push_back(floats);
    scratch.push_back(nullptr);
    return int(scratch.size() - 1);
  }
  static size_t slot(size_t floats) { return (floats + 63) / 64 * 64; }  // 256-byte aligned slots
  size_t scratch_total() const {
    size_t t = 0;
    for (size_t f : scratch_floats) t += slot(f);
    return t;
  }
  void place_scratch(float* base) {
    for (size_t k = 0; k < scratch.size(); ++k) {
      scratch[k] = base;
      base += slot(scratch_floats[k]);
    }
  }
  int materialise(const Node* n);
  int stab_grad(const Node* operand);
  // stab stage-1 passes not yet emitted: (operand: a field, a scratch buffer
  // or an inline node; output scratch).  They are merged into one kernel,
  // emitted before the next pass that may read them.
  struct PendingStab {
    JitInput src;
    const Node* node;  // inline operand, else null
    int out;
  };
  std::vector<PendingStab> pending_stab;
  bool flushing = false;
  void flush_stab();
  void add_pass(const std::string& src, const char* entry, std::vector<JitInput> inputs, int out) {
    flush_stab();
    auto p = std::make_unique<JitPass>();
    p->source = src;
    p->entry = entry;
    p->inputs = std::move(inputs);
    p->out_scratch = out;
    passes.push_back(std::move(p));
  }
};

// One generated kernel.
struct JitGen {
  JitPlan& plan;
  std::vector<JitInput> inputs;
  std::map<const Node*, int> done;
  std::string funcs;
  int next = 0;
  // in a group kernel: fields written by earlier members -> their slot in V
  // (the member's value at this cell, held in a register)
  const std::map<Variable*, int>* written = nullptr;
  explicit JitGen(JitPlan& p) : plan(p) {}

  static std::string lit(float v) {
    uint32_t bits;
    std::memcpy(&bits, &v, sizeof(bits));
    char b[48];
    std::snprintf(b, sizeof(b), "__uint_as_float(0x%08xu)", bits);
    return b;
  }
  int input(const JitInput& in) {
    for (size_t k = 0; k < inputs.size(); ++k)
      if (inputs[k] == in) return int(k);
    inputs.push_back(in);
    return int(inputs.size() - 1);
  }
  // an expression of fields, constants and dt alone (evaluated at any cell inline)
  static bool pointwise(const Node* n, int* budget) {
    if (--*budget < 0) return false;
    switch (n->kind) {
      case Node::kField:
      case Node::kConst:
      case Node::kDt: return true;
      case Node::kBinary: return pointwise(n->a.get(), budget) && pointwise(n->b.get(), budget);
      case Node::kNeg: return pointwise(n->a.get(), budget);
      default: return false;
    }
  }
  static bool inline_operand(const Node* n) {
    int budget = 48;
    return pointwise(n, &budget);
  }
  // operand of a neighbour operator as a callable of the cell index: a
  // field's buffer, a pointwise expression evaluated inline, or the buffer an
  // earlier pass materialised it into
  std::string operand(const Node* n) {
    if (n->kind == Node::kField)
      return "[&](long long j) { return A.f[" + std::to_string(input(JitInput{n->field, -1})) + "][j]; }";
    if (inline_operand(n)) {
      const int k = emit(n);
      if (k < 0) return std::string();
      return "[&](long long j) { return e" + std::to_string(k) + "(j, A, V); }";
    }
    const int s = plan.materialise(n);
    if (s < 0) return std::string();
    return "[&](long long j) { return A.f[" + std::to_string(input(JitInput{nullptr, s})) + "][j]; }";
  }
  std::string call(int k) { return "e" + std::to_string(k) + "(i, A, V)"; }
  int emit(const Node* n) {
    auto it = done.find(n);
    if (it != done.end()) return it->second;
    if (!plan.ok) return -1;
    std::string body;
    static const char* ops[] = {" + ", " - ", " * ", " / "};
    switch (n->kind) {
      case Node::kField: {
        auto w = written ? written->find(n->field) : std::map<Variable*, int>::const_iterator();
        if (written && w != written->end()) body = "V[" + std::to_string(w->second) + "]";
        else body = "A.f[" + std::to_string(input(JitInput{n->field, -1})) + "][i]";
        break;
      }
      case Node::kConst: body = lit(n->value); break;
      case Node::kDt: body = "A.dt"; break;
      case Node::kBinary: {
        if (n->op < 0 || n->op > 3) {
          plan.ok = false;
          return -1;
        }
        const int a = emit(n->a.get()), b = emit(n->b.get());
        if (a < 0 || b < 0) return -1;
        body = call(a) + ops[n->op] + call(b);
        break;
      }
      case Node::kNeg: {
        const int a = emit(n->a.get());
        if (a < 0) return -1;
        body = "-" + call(a);
        break;
      }
      case Node::kGrad:
      case Node::kLapl: {
        const std::string phi = operand(n->a.get());
        if (!plan.ok || phi.empty()) return -1;
        body = std::string(n->kind == Node::kGrad ? "cfdb_grad" : "cfdb_lapl") + "(" + phi + ", i, " +
               std::to_string(n->mask) + ", A.g)";
        break;
      }
      case Node::kStab: {
        const int gr = plan.stab_grad(n->a.get());
        if (!plan.ok || gr < 0) return -1;
        const std::string phi = operand(n->a.get());
        if (!plan.ok || phi.empty()) return -1;
        body = "cfdb_stab2g(" + phi + ", A.f[" + std::to_string(input(JitInput{nullptr, gr})) + "], i, " +
               std::to_string(n->mask) + ", A.g)";
        break;
      }
      default:
        plan.ok = false;
        return -1;
    }
    const int k = next++;
    funcs += "__device__ __forceinline__ float e" + std::to_string(k) +
             "(long long i, const CfdbArgs& A, const float* V) { return " + body + "; }\n";
    done[n] = k;
    return k;
  }
  std::string prelude() const {
    return "#include \"cfdb_jit.cuh\"\n" + plan.lattice_struct() + "struct CfdbArgs { const float* f[" +
           std::to_string(std::max<size_t>(1, inputs.size())) + "]; float dt; " + plan.geom_type() + " g; };\n";
  }
  // every generated kernel has the signature (A, out, cur, prev, mode, n)
  std::string equation_source(int root) const {
    return prelude() + funcs +
           "extern \"C\" __global__ void cfdb_equation(CfdbArgs A, float* __restrict__ out, const float* __restrict__ cur,\n"
           "                                        const float* __restrict__ prev, int mode, long long n) {\n"
           "  const float* V = nullptr;\n" +
           JitPlan::cells(kCptEquation, "  float Rv[" + std::to_string(kCptEquation) + "];\n",
                          "      Rv[c] = e" + std::to_string(root) + "(i, A, V);\n",
                          "      const float R = Rv[c];\n"
                          "      if (mode == 0) out[i] = R;                                  // plain left-hand side, scratch\n"
                          "      else if (mode == 1) out[i] = A.dt * R + cur[i];             // d1t, first d2t step\n"
                          "      else out[i] = (A.dt * A.dt * R + 2.0f * cur[i]) - prev[i];  // d2t\n") +
           "}\n";
  }
};

int JitPlan::materialise(const Node* n) {
  auto it = materialised.find(n);
  if (it != materialised.end()) return it->second;
  JitGen g(*this);
  const int root = g.emit(n);
  if (!ok || root < 0) {
    ok = false;
    return -1;
  }
  const int s = new_scratch(mesh->_num_nodes);
  add_pass(g.equation_source(root), "cfdb_equation", g.inputs, s);
  passes.back()->cpt = kCptEquation;
  materialised[n] = s;
  return s;
}

// Stage 1 of a stabilisation: the operand's three gradient components per
// cell into a 3n scratch, one per distinct operand (a field, or an operand
// node); the kernel is emitted later, merged with the plan's other stage-1
// passes (flush_stab).  An operand that holds operators is materialised now.
int JitPlan::stab_grad(const Node* operand) {
  const void* key = operand->kind == Node::kField ? static_cast<const void*>(operand->field) : operand;
  auto it = stab_grads.find(key);
  if (it != stab_grads.end()) return it->second;
  PendingStab ps{};
  if (operand->kind == Node::kField) {
    ps.src = JitInput{operand->field, -1};
  } else if (JitGen::inline_operand(operand)) {
    ps.node = operand;
  } else {
    const int m = materialise(operand);
    if (m < 0) {
      ok = false;
      return -1;
    }
    ps.src = JitInput{nullptr, m};
  }
  ps.out = new_scratch(3 * mesh->_num_nodes);
  pending_stab.push_back(ps);
  stab_grads[key] = ps.out;
  return ps.out;
}

// Emits the pending stage-1 passes, one kernel per operand.  (One kernel for
// all of them, sharing the loads of common fields, measured 1.3x slower on
// the reference's Euler system at 200^3: fewer resident warps, no reuse won.)
void JitPlan::flush_stab() {
  if (pending_stab.empty() || flushing) return;
  if (pending_stab.size() > 1) {  // one kernel per operand (measured faster than one merged kernel)
    const auto all = pending_stab;
    for (const auto& ps : all) {
      pending_stab.assign(1, ps);
      flush_stab();
    }
    return;
  }
  flushing = true;
  JitGen g(*this);
  std::string body, stores;
  std::vector<JitInput> outs;
  for (const PendingStab& ps : pending_stab) {
    const std::string phi =
        ps.node ? g.operand(ps.node)
                : "[&](long long j) { return A.f[" + std::to_string(g.input(ps.src)) + "][j]; }";
    if (!ok || phi.empty()) {
      ok = false;
      break;
    }
    const std::string k = std::to_string(outs.size());
    for (int d = 0; d < 3; ++d) {  // the components cfdb_stab_grad stores, each at d*n + i of its buffer
      const std::string slot = std::to_string(3 * outs.size() + size_t(d));
      body += "      G[c][" + slot + "] = cfdb_grad_component(" + phi + ", i, " + std::to_string(d) + ", A.g);\n";
      stores += "      A.o[" + k + "][" + std::to_string(d) + " * n + i] = G[c][" + slot + "];\n";
    }
    outs.push_back(JitInput{nullptr, ps.out});
  }
  pending_stab.clear();
  if (ok) {
    const std::string src =
        "#include \"cfdb_jit.cuh\"\n" + lattice_struct() + "struct CfdbArgs { const float* f[" +
        std::to_string(std::max<size_t>(1, g.inputs.size())) + "]; float* o[" + std::to_string(outs.size()) +
        "]; float dt; " + geom_type() + " g; };\n" + g.funcs +
        "extern \"C\" __global__ void cfdb_stab_stage1(CfdbArgs A, long long n) {\n"
        "  const float* V = nullptr;\n" +
        cells(kCptStab, "  float G[" + std::to_string(kCptStab) + "][" + std::to_string(3 * outs.size()) + "];\n",
              body, stores) +
        "}\n";
    add_pass(src, "cfdb_stab_stage1", g.inputs, -1);
    passes.back()->multi = true;
    passes.back()->outputs = outs;
    passes.back()->cpt = kCptStab;
  }
  flushing = false;
}

std::unique_ptr<JitPlan> new_plan(Mesh3D* mesh) {
  auto plan = std::make_unique<JitPlan>();
  plan->mesh = mesh;
  if (CFDArcoGlobalInit::jit_lattice) {
    check(cfdb_mesh_lattice_geometry(mesh->handle(), &plan->lat), "cfdb_mesh_lattice_geometry");
    plan->lattice = plan->lat.exact != 0;
    for (const float* v = plan->lat.normal; v <= &plan->lat.volume; ++v) plan->lattice = plan->lattice && std::isfinite(*v);
  }
  return plan;
}

std::unique_ptr<JitPlan> jit_build(const Node* rhs, Mesh3D* mesh) {
  auto plan = new_plan(mesh);
  JitGen g(*plan);
  const int root = g.emit(rhs);
  if (!plan->ok || root < 0) return nullptr;
  plan->add_pass(g.equation_source(root), "cfdb_equation", g.inputs, -1);
  plan->passes.back()->cpt = kCptEquation;
  return plan;
}

// Fields an expression reads inside the operand of a neighbour operator
// (grad, lapl, stab: at other cells, or in a pass of their own) and the ones
// it reads at its own cell only.
void collect_fields(const Node* n, bool in_operand, std::set<Variable*>& nb, std::set<Variable*>& own) {
  switch (n->kind) {
    case Node::kField: (in_operand ? nb : own).insert(n->field); break;
    case Node::kBinary:
      collect_fields(n->a.get(), in_operand, nb, own);
      collect_fields(n->b.get(), in_operand, nb, own);
      break;
    case Node::kNeg: collect_fields(n->a.get(), in_operand, nb, own); break;
    case Node::kGrad:
    case Node::kLapl:
    case Node::kStab: collect_fields(n->a.get(), true, nb, own); break;
    default: break;
  }
}

// One member of a group: the equation's right-hand side, the field it
// writes and its form (0 plain left-hand side, 1 d1t).
struct GroupMember {
  const Node* rhs;
  Variable* target;
  int form;
};

// A run of consecutive equations compiled into one kernel (after the
// pre-passes their operands need).  Every member's right-hand side is
// evaluated in order at the thread's cell; a field written by an earlier
// member is read from that member's register value (the equations run in
// sequence, so the later ones see it updated), and no member reads such a
// field at another cell (the caller ends a group before that would happen).
// Each written field's last value goes to its next buffer.  Arithmetic per
// member is that of the single-equation kernel, so the bits are the same.
std::unique_ptr<JitPlan> jit_group_build(const std::vector<GroupMember>& members, Mesh3D* mesh) {
  auto plan = new_plan(mesh);
  JitGen g(*plan);
  std::map<Variable*, int> written;
  std::string body;
  for (size_t m = 0; m < members.size(); ++m) {
    const GroupMember& gm = members[m];
    g.done.clear();  // a node's value may differ once an earlier member wrote one of its fields
    g.written = &written;
    const int root = g.emit(gm.rhs);
    if (!plan->ok || root < 0) return nullptr;
    std::string update = "R";
    if (gm.form == 1) {
      auto w = written.find(gm.target);
      const std::string cur = w != written.end() ? "V[" + std::to_string(w->second) + "]"
                                                 : "A.f[" + std::to_string(g.input(JitInput{gm.target, -1})) + "][i]";
      update = "A.dt * R + " + cur;
    }
    body += "      { const float R = e" + std::to_string(root) + "(i, A, V); V[" + std::to_string(m) + "] = " + update +
            "; }\n";
    written[gm.target] = int(m);
  }
  std::vector<Variable*> outputs;
  std::string stores;
  for (const auto& kv : written) {
    stores += "      A.o[" + std::to_string(outputs.size()) + "][i] = VV[c][" + std::to_string(kv.second) + "];\n";
    outputs.push_back(kv.first);
  }
  const std::string src =
      "#include \"cfdb_jit.cuh\"\n" + plan->lattice_struct() + "struct CfdbArgs { const float* f[" +
      std::to_string(std::max<size_t>(1, g.inputs.size())) + "]; float* o[" + std::to_string(outputs.size()) +
      "]; float dt; " + plan->geom_type() + " g; };\n" + g.funcs +
      "extern \"C\" __global__ void cfdb_group(CfdbArgs A, long long n) {\n" +
      JitPlan::cells(kCptGroup,
                     "  float VV[" + std::to_string(kCptGroup) + "][" + std::to_string(members.size()) + "];\n",
                     "      float* V = VV[c];\n" + body, stores) +
      "}\n";
  plan->add_pass(src, "cfdb_group", g.inputs, -1);
  plan->passes.back()->cpt = kCptGroup;
  plan->passes.back()->multi = true;
  for (Variable* v : outputs) plan->passes.back()->outputs.push_back(JitInput{v, -1});
  return plan;
}

// KernelBuilder::build for every plan of an equation system in one call: the
// library compiles the sources on several host threads (or loads them from
// its on-disk kernel cache).
void jit_compile(const std::vector<std::unique_ptr<JitPlan>*>& plans) {
  std::vector<JitPass*> passes;
  for (const auto* plan : plans)
    if (*plan)
      for (const auto& p : (*plan)->passes)
        if (!p->k) passes.push_back(p.get());
  if (passes.empty()) return;
  std::vector<const char*> srcs, names;
  for (JitPass* p : passes) {
    srcs.push_back(p->source.c_str());
    names.push_back(p->entry.c_str());
  }
  std::vector<cfdb_kernel*> ks(passes.size(), nullptr);
  check(cfdb_kernel_build_many(CFDArcoGlobalInit::ctx(), int(passes.size()), srcs.data(), names.data(), ks.data()),
        "cfdb_kernel_build_many");
  for (size_t k = 0; k < passes.size(); ++k) {
    passes[k]->k = ks[k];
    if (CFDArcoGlobalInit::jit_report) {
      int regs = 0, maxt = 0;
      int64_t local = 0;
      check(cfdb_kernel_info(ks[k], &regs, &local, &maxt), "cfdb_kernel_info");
      std::fprintf(stderr, "jit kernel %zu: %s, %d registers, %lld local bytes, %d cells per thread\n", k,
                   passes[k]->entry.c_str(), regs, (long long)local, passes[k]->cpt);
    }
  }
}

// KernelBuilder::run: the plan's passes in order; the last one writes the
// equation's update (mode 0: value, 1: d1t, 2: d2t) into `out`.
void jit_run(const JitPlan& plan, float dt, float* out, const float* cur, const float* prev, int mode) {
  // CfdbArgs { const float* f[nf]; float dt; G g; } laid out as the device
  // compiler does: G = CfdbGeom (pointers, 8-byte aligned) or the empty
  // CfdbLattice<CfdbC>; the struct's size rounds up to its 8-byte alignment
  struct Geom {
    const int32_t* ids;
    const float *normal, *normal_alt, *area, *alpha, *len, *volume;
    long long n;
  } geom{};
  const unsigned char* gsrc;
  size_t gsize, galign;
  static const unsigned char empty = 0;
  if (plan.lattice) {  // CfdbLattice<CfdbC> is an empty struct: its constants are in the source
    gsrc = &empty;
    gsize = 1;
    galign = 1;
  } else {
    cfdb_plain_geometry g{};
    check(cfdb_mesh_plain_geometry(plan.mesh->handle(), &g), "cfdb_mesh_plain_geometry");
    geom = Geom{g.ids, g.normal, g.normal_alt, g.area, g.alpha, g.len, g.volume, (long long)g.n};
    gsrc = reinterpret_cast<const unsigned char*>(&geom);
    gsize = sizeof(geom);
    galign = alignof(Geom);
  }
  long long n = (long long)plan.mesh->_num_nodes;
  for (const auto& p : plan.passes) {
    // group passes carry their output pointers after the inputs: { f[nf]; o[no]; dt; g }
    const size_t nf = std::max<size_t>(1, p->inputs.size()), no = p->multi ? p->outputs.size() : 0;
    const size_t off_dt = (nf + no) * sizeof(void*);
    const size_t off_g = (off_dt + sizeof(float) + galign - 1) / galign * galign;
    std::vector<unsigned char> A((off_g + gsize + 7) / 8 * 8, 0);
    for (size_t k = 0; k < p->inputs.size(); ++k) {
      const JitInput& in = p->inputs[k];
      const float* ptr = in.field ? in.field->current_cu : plan.scratch[size_t(in.scratch)];
      std::memcpy(&A[k * sizeof(void*)], &ptr, sizeof(ptr));
    }
    for (size_t k = 0; k < no; ++k) {
      const JitInput& o = p->outputs[k];
      float* ptr = o.field ? o.field->next_cu : plan.scratch[size_t(o.scratch)];
      std::memcpy(&A[(nf + k) * sizeof(void*)], &ptr, sizeof(ptr));
    }
    std::memcpy(&A[off_dt], &dt, sizeof(dt));
    std::memcpy(&A[off_g], gsrc, gsize);
    // cpt cells per thread: chunks of 256 cells, one CTA per 256 * cpt cells
    const long long blocks = (n + 256LL * p->cpt - 1) / (256LL * p->cpt);
    if (p->multi) {
      void* args[] = {A.data(), &n};
      check(cfdb_kernel_launch(p->k, blocks * 256, 256, args), "cfdb_kernel_launch");
      continue;
    }
    float* o = p->out_scratch >= 0 ? plan.scratch[size_t(p->out_scratch)] : out;
    int m = p->out_scratch >= 0 ? 0 : mode;
    void* args[] = {A.data(), &o, &cur, &prev, &m, &n};
    check(cfdb_kernel_launch(p->k, blocks * 256, 256, args), "cfdb_kernel_launch");
  }
}

// Whether the fused TMA step can serve this mesh (uniform, z rows of 16 bytes).
bool stencil_fusable(Mesh3D* mesh) {
  int64_t dims[3];
  double h[3];
  int uniform = 0;
  check(cfdb_mesh_info(mesh->handle(), dims, h, &uniform), "cfdb_mesh_info");
  return uniform && dims[2] % 4 == 0;
}

// k * lapl(T) or lapl(T) * k or lapl(T) with T the updated field: the heat
// template that runs as one fused step.
bool match_heat(const Node* rhs, const Variable* T, float* k) {
  auto is_lapl_T = [&](const Node* n) {
    return n->kind == Node::kLapl && n->mask == 7 && n->a->kind == Node::kField && n->a->field == T;
  };
  if (is_lapl_T(rhs)) {
    *k = 1.f;
    return true;
  }
  if (rhs->kind == Node::kBinary && rhs->op == CFDB_OP_MUL) {
    if (rhs->a->kind == Node::kConst && is_lapl_T(rhs->b.get())) {
      *k = rhs->a->value;
      return true;
    }
    if (rhs->b->kind == Node::kConst && is_lapl_T(rhs->a.get())) {
      *k = rhs->b->value;
      return true;
    }
  }
  return false;
}

// d2t(u) = k * S, S * k or S, with S Laplacians of u (d2dx, d2dy, d2dz,
// lapl, ...) summed left to right, at most three: the wave template that
// cfdb_d2t_step runs as one fused pass with the generated kernel's rounding.
struct D2tForm {
  float k = 1.f;
  int32_t masks[3] = {0, 0, 0};
  int32_t n = 0;
};
bool match_d2t(const Node* rhs, const Variable* u, D2tForm* out) {
  D2tForm f;
  const Node* sum = rhs;
  if (rhs->kind == Node::kBinary && rhs->op == CFDB_OP_MUL) {
    if (rhs->a->kind == Node::kConst) {
      f.k = rhs->a->value;
      sum = rhs->b.get();
    } else if (rhs->b->kind == Node::kConst) {
      f.k = rhs->b->value;
      sum = rhs->a.get();
    }
  }
  auto lapl_u = [&](const Node* n) {
    return n->kind == Node::kLapl && n->mask >= 1 && n->mask <= 7 && n->a->kind == Node::kField && n->a->field == u;
  };
  std::vector<int32_t> masks;
  const Node* n = sum;
  while (n->kind == Node::kBinary && n->op == CFDB_OP_ADD && lapl_u(n->b.get())) {
    masks.insert(masks.begin(), n->b->mask);
    n = n->a.get();
  }
  if (!lapl_u(n)) return false;
  masks.insert(masks.begin(), n->mask);
  if (masks.size() > 3) return false;
  for (size_t j = 0; j < masks.size(); ++j) f.masks[j] = masks[j];
  f.n = int32_t(masks.size());
  *out = f;
  return true;
}

// The mesh is an exact lattice (per-slot geometry constants, all finite).
bool lattice_exact(Mesh3D* mesh) {
  cfdb_lattice_geometry lat{};
  check(cfdb_mesh_lattice_geometry(mesh->handle(), &lat), "cfdb_mesh_lattice_geometry");
  bool ok = lat.exact != 0;
  for (const float* v = lat.normal; v <= &lat.volume; ++v) ok = ok && std::isfinite(*v);
  return ok;
}

}  // namespace

// ---------------------------------------------------------------------------
// Variable
// ---------------------------------------------------------------------------
Variable::Variable() = default;

Variable::Variable(Mesh3D* m, HostVec& initial, BoundaryFN bc, std::string nm)
    : name(std::move(nm)), mesh(m), current(initial), boundary_conditions(std::move(bc)), is_field(true) {
  if (initial.size() != m->_num_nodes) throw std::runtime_error("Variable: initial values do not match the mesh");
  node = make(Node::kField, m);
  node->field = this;
  current_cu = device_alloc(m->_num_nodes);
  next_cu = device_alloc(m->_num_nodes);
  check(cfdb_upload(CFDArcoGlobalInit::ctx(), current_cu, initial.data(), int64_t(initial.size() * sizeof(float))),
        "cfdb_upload");
}

Variable::Variable(Mesh3D* m, HostVec& initial, BoundaryFN bc, BoundaryFNCU bc_cu, std::string nm)
    : Variable(m, initial, std::move(bc), std::move(nm)) {
  boundary_conditions_cu = std::move(bc_cu);
  has_boundary_conditions_cu = bool(boundary_conditions_cu);
}

Variable::Variable(Mesh3D* m, float value) : mesh(m) {
  node = make(Node::kConst, m);
  node->value = value;
  name = "const";
}

Variable::~Variable() {
  if (is_field && node && node->field == this) {
    device_free(current_cu);
    device_free(next_cu);
    device_free(prev_cu);
    node->field = nullptr;
  }
}

const HostVec& Variable::host() {
  if (is_field) {
    current.resize(mesh->_num_nodes);
    check(cfdb_download(CFDArcoGlobalInit::ctx(), current.data(), current_cu, int64_t(current.size() * sizeof(float))),
          "cfdb_download");
  }
  return current;
}

void Variable::set_current(const HostVec& values) {
  current = values;
  check(cfdb_upload(CFDArcoGlobalInit::ctx(), current_cu, values.data(), int64_t(values.size() * sizeof(float))),
        "cfdb_upload");
}

Variable Variable::operator+(const Variable& r) const { return binary(*this, r, CFDB_OP_ADD); }
Variable Variable::operator-(const Variable& r) const { return binary(*this, r, CFDB_OP_SUB); }
Variable Variable::operator*(const Variable& r) const { return binary(*this, r, CFDB_OP_MUL); }
Variable Variable::operator/(const Variable& r) const { return binary(*this, r, CFDB_OP_DIV); }
Variable Variable::operator-() const {
  auto n = make(Node::kNeg, mesh);
  n->a = node;
  return wrap(n);
}

Variable operator+(float l, const Variable& r) { return Variable(r.mesh, l) + r; }
Variable operator-(float l, const Variable& r) { return Variable(r.mesh, l) - r; }
Variable operator*(float l, const Variable& r) { return Variable(r.mesh, l) * r; }
Variable operator/(float l, const Variable& r) { return Variable(r.mesh, l) / r; }
Variable operator+(const Variable& l, float r) { return l + Variable(l.mesh, r); }
Variable operator-(const Variable& l, float r) { return l - Variable(l.mesh, r); }
Variable operator*(const Variable& l, float r) { return l * Variable(l.mesh, r); }
Variable operator/(const Variable& l, float r) { return l / Variable(l.mesh, r); }

namespace {
std::vector<std::unique_ptr<Variable>>& lhs_registry() {
  static std::vector<std::unique_ptr<Variable>> r;
  return r;
}
}  // namespace

DtVar* d1t(Variable& v) {
  auto* d = new DtVar(&v);
  d->name = "d1t(" + v.name + ")";
  lhs_registry().emplace_back(d);
  return d;
}

D2tVar* d2t(Variable& v) {
  auto* d = new D2tVar(&v);
  d->name = "d2t(" + v.name + ")";
  lhs_registry().emplace_back(d);
  return d;
}

Variable d1dx(const Variable& v) { return mesh_op(v, Node::kGrad, 1); }
Variable d1dy(const Variable& v) { return mesh_op(v, Node::kGrad, 2); }
Variable d1dz(const Variable& v) { return mesh_op(v, Node::kGrad, 4); }
Variable d2dx(const Variable& v) { return mesh_op(v, Node::kLapl, 1); }
Variable d2dy(const Variable& v) { return mesh_op(v, Node::kLapl, 2); }
Variable d2dz(const Variable& v) { return mesh_op(v, Node::kLapl, 4); }
Variable lapl(const Variable& v) { return mesh_op(v, Node::kLapl, 7); }
Variable stab_tot(const Variable& v) { return mesh_op(v, Node::kStab, 7); }
Variable stabx(const Variable& v) { return mesh_op(v, Node::kStab, 1); }
Variable staby(const Variable& v) { return mesh_op(v, Node::kStab, 2); }
Variable stabz(const Variable& v) { return mesh_op(v, Node::kStab, 4); }

HostVec boundary_none(Mesh3D*, HostVec& arr, const DT*) { return arr; }

namespace {
// The boundary copy as a callable the time loop can recognise: a heat
// equation whose field has it runs the copy inside its fused step.
struct BoundaryCopyCu {
  std::shared_ptr<float> buf;
  size_t count = 0;
  // in place over the boundary cells only (the reference's blend
  // arr * (1 - b) + copy * b leaves the interior as it is for finite states)
  void operator()(Mesh3D* m, float* field, const DT*) const {
    check(cfdb_op_boundary_set(CFDArcoGlobalInit::ctx(), m->handle(), CFDB_F32, field, buf.get()),
          "cfdb_op_boundary_set");
  }
};
}  // namespace

BoundaryFNCU boundary_copy_cu(Mesh3D* mesh, const HostVec& values) {
  auto buf = std::shared_ptr<float>(device_alloc(values.size()), [](float* p) { device_free(p); });
  check(cfdb_upload(CFDArcoGlobalInit::ctx(), buf.get(), values.data(), int64_t(values.size() * sizeof(float))),
        "cfdb_upload");
  return BoundaryCopyCu{buf, values.size()};
}

// ---------------------------------------------------------------------------
// DT and the update policies
// ---------------------------------------------------------------------------
DT::DT(Mesh3D* m, UpdateFn fn, float cfl, std::vector<Variable*> vars)
    : update_fn(std::move(fn)), CFL(cfl), space_vars(std::move(vars)) {
  mesh = m;
  name = "dt";
  node = make(Node::kDt, m);
  node->dt = this;
}

void DT::update() {
  _dt = update_fn(CFL, space_vars, mesh);
  ++_current_time_step_int;
  _current_time_dbl += _dt;
}

float UpdatePolicies::CourantFriedrichsLewy3D(float CFL, std::vector<Variable*>& v, Mesh3D* mesh) {
  double dt = 0;
  check(cfdb_cfl_dt(CFDArcoGlobalInit::ctx(), mesh->handle(), CFDB_F32, CFL, 5.0 / 3.0, v.at(3)->current_cu,
                    v.at(4)->current_cu, v.at(0)->current_cu, v.at(1)->current_cu, v.at(2)->current_cu, &dt),
        "cfdb_cfl_dt");
  return float(dt);
}

float UpdatePolicies::CourantFriedrichsLewy1D(float CFL, std::vector<Variable*>& v, Mesh3D* mesh) {
  double dt = 0;
  check(cfdb_cfl_dt(CFDArcoGlobalInit::ctx(), mesh->handle(), CFDB_F32, CFL, 5.0 / 3.0, v.at(1)->current_cu,
                    v.at(2)->current_cu, v.at(0)->current_cu, nullptr, nullptr, &dt),
        "cfdb_cfl_dt");
  return float(dt);
}

// ---------------------------------------------------------------------------
// Equation
// ---------------------------------------------------------------------------
Equation::Equation(size_t t) : timesteps(t) {}

void Equation::evaluate(std::vector<Variable*>& all_vars, EquationTemplate& eqs, DT* dt, bool visualize,
                        std::vector<Variable*> store_vars) const {
  cfdb_ctx* ctx = CFDArcoGlobalInit::ctx();
  // phase times on the host clock, printed with jit_report
  using Clock = std::chrono::steady_clock;
  const auto t_start = Clock::now();
  auto ms_since = [](Clock::time_point a) { return std::chrono::duration<double, std::milli>(Clock::now() - a).count(); };
  double ms_plan = 0, ms_compile = 0, ms_first = 0;
  fused_equations = 0;
  jit_equations = 0;
  lattice_equations = 0;
  jit_groups = 0;
  // use_jit equations (tuple element 3), and with jit_all the others too,
  // that are not the fused heat template run as generated kernels, all
  // compiled before the first step: consecutive plain and d1t equations fuse
  // into groups (one kernel after their operands' pre-passes), a group ending
  // where a member would read at other cells a field an earlier member wrote;
  // d2t equations get a plan of their own.
  struct Unit {
    std::unique_ptr<JitPlan> plan;
    size_t count = 1;    // equations the unit covers, from its first
    bool group = false;
  };
  std::vector<Unit> units;
  std::vector<int> unit_at(eqs.size(), -1);  // unit starting at this equation
  std::map<size_t, D2tForm> fused_d2t;       // d2t equations run by cfdb_d2t_step
  std::vector<GroupMember> open;
  size_t open_first = 0;
  Mesh3D* open_mesh = nullptr;
  std::set<Variable*> open_written;
  auto close_group = [&] {
    if (open.empty()) return;
    auto plan = jit_group_build(open, open_mesh);
    if (plan) {  // otherwise the members stay on the operator path
      jit_equations += int(open.size());
      if (plan->lattice) lattice_equations += int(open.size());
      ++jit_groups;
      unit_at[open_first] = int(units.size());
      units.push_back(Unit{std::move(plan), open.size(), true});
    }
    open.clear();
    open_written.clear();
  };
  jit_groups = 0;
  constexpr size_t kMaxGroup = 16;
  for (size_t e = 0; e < eqs.size(); ++e) {
    Variable* lhs = std::get<0>(eqs[e]);
    const Node* rhs = std::get<2>(eqs[e]).node.get();
    float k = 0.f;
    auto* d = dynamic_cast<DtVar*>(lhs);
    auto* d2 = dynamic_cast<D2tVar*>(lhs);
    Mesh3D* mesh = d ? d->var->mesh : (d2 ? d2->var->mesh : lhs->mesh);
    const bool generate = rhs && mesh && (std::get<3>(eqs[e]) || CFDArcoGlobalInit::jit_all) &&
                          !(d && match_heat(rhs, d->var, &k) && stencil_fusable(d->var->mesh)) &&
                          (d || d2 || lhs->is_field);
    if (!generate) {
      close_group();
      continue;
    }
    if (d2) {
      close_group();
      // the wave template on an exact lattice: one fused pass instead of a
      // generated kernel (the face-array form, jit_lattice off, keeps the latter)
      D2tForm form;
      if (CFDArcoGlobalInit::jit_lattice && match_d2t(rhs, d2->var, &form) && stencil_fusable(mesh) &&
          lattice_exact(mesh)) {
        fused_d2t[e] = form;
        continue;
      }
      auto plan = jit_build(rhs, mesh);
      if (plan) {
        ++jit_equations;
        if (plan->lattice) ++lattice_equations;
        unit_at[e] = int(units.size());
        units.push_back(Unit{std::move(plan), 1, false});
      }
      continue;
    }
    std::set<Variable*> nb, own;
    collect_fields(rhs, false, nb, own);
    bool clash = mesh != open_mesh || open.size() >= kMaxGroup;
    for (Variable* v : nb) clash = clash || open_written.count(v) > 0;
    if (clash) close_group();
    if (open.empty()) {
      open_first = e;
      open_mesh = mesh;
    }
    Variable* target = d ? d->var : lhs;
    open.push_back(GroupMember{rhs, target, d ? 1 : 0});
    open_written.insert(target);
  }
  close_group();
  // every plan's scratch in one block, returned when evaluate ends
  struct Block {
    float* p = nullptr;
    ~Block() { device_free(p); }
  } scratch;
  {
    size_t total = 0;
    for (Unit& u : units) total += u.plan->scratch_total();
    if (total) scratch.p = device_alloc(total);
    float* at = scratch.p;
    for (Unit& u : units) {
      u.plan->place_scratch(at);
      at += u.plan->scratch_total();
    }
  }
  ms_plan = ms_since(t_start);
  {
    std::vector<std::unique_ptr<JitPlan>*> plans;
    for (Unit& u : units) plans.push_back(&u.plan);
    jit_compile(plans);
  }
  ms_compile = ms_since(t_start) - ms_plan;
  for (size_t t = 0; t < timesteps; ++t) {
    Variable* bc_done = nullptr;  // a field whose boundary copy ran inside its fused step
    if (t == 1 && CFDArcoGlobalInit::jit_report) {
      check(cfdb_sync(ctx), "cfdb_sync");
      ms_first = ms_since(t_start) - ms_plan - ms_compile;
    }
    dt->update();
    const float dtv = dt->_dt;
    for (size_t e = 0; e < eqs.size(); ++e) {
      auto& eq = eqs[e];
      Variable* lhs = std::get<0>(eq);
      Variable& rhs = std::get<2>(eq);
      const Unit* U = unit_at[e] >= 0 ? &units[size_t(unit_at[e])] : nullptr;
      if (U && U->group) {
        jit_run(*U->plan, dtv, nullptr, nullptr, nullptr, 0);
        for (const JitInput& o : U->plan->passes.back()->outputs) std::swap(o.field->current_cu, o.field->next_cu);
        e += U->count - 1;
        continue;
      }
      const JitPlan* J = U ? U->plan.get() : nullptr;
      if (auto* d = dynamic_cast<DtVar*>(lhs)) {
        Variable* T = d->var;
        const int64_t N = int64_t(T->mesh->_num_nodes);
        float k = 0.f;
        // a one-equation, one-field system whose field resets its surface
        // cells to a copy after each step: the copy runs inside the fused
        // step (no other boundary function can observe the difference)
        const BoundaryCopyCu* copy = nullptr;
        if (eqs.size() == 1 && all_vars.size() == 1 && all_vars[0] == T && T->has_boundary_conditions_cu) {
          copy = T->boundary_conditions_cu.target<BoundaryCopyCu>();
          if (copy && copy->count != size_t(N)) copy = nullptr;
        }
        if (copy && match_heat(rhs.node.get(), T, &k) &&
            cfdb_heat_step_fixed(ctx, T->mesh->handle(), CFDB_F32, T->current_cu, T->next_cu, k, dtv,
                                 copy->buf.get()) == CFDB_OK) {
          if (t == 0) ++fused_equations;
          bc_done = T;
        } else if (match_heat(rhs.node.get(), T, &k) &&
                   cfdb_heat_step(ctx, T->mesh->handle(), CFDB_F32, CFDB_PATH_FUSED, T->current_cu, T->next_cu, k,
                                  dtv) == CFDB_OK) {
          if (t == 0) ++fused_equations;
        } else {
          const float* R = eval_node(rhs.node.get());
          check(cfdb_op_d1t(ctx, CFDB_F32, R, T->current_cu, dtv, T->next_cu, N), "cfdb_op_d1t");
        }
        std::swap(T->current_cu, T->next_cu);
      } else if (auto* d2 = dynamic_cast<D2tVar*>(lhs)) {
        Variable* Uv = d2->var;
        const int64_t N = int64_t(Uv->mesh->_num_nodes);
        if (!Uv->prev_cu) Uv->prev_cu = device_alloc(Uv->mesh->_num_nodes);
        auto fz = fused_d2t.find(e);
        if (fz != fused_d2t.end()) {
          const D2tForm& f = fz->second;
          check(cfdb_d2t_step(ctx, Uv->mesh->handle(), CFDB_F32, Uv->current_cu, Uv->has_prev ? Uv->prev_cu : nullptr,
                              Uv->next_cu, f.k, f.masks, f.n, dtv, Uv->has_prev ? 0 : 1),
                "cfdb_d2t_step");
          if (t == 0) ++fused_equations;
        } else if (J) {
          jit_run(*J, dtv, Uv->next_cu, Uv->current_cu, Uv->prev_cu, Uv->has_prev ? 2 : 1);
        } else {
          const float* R = eval_node(rhs.node.get());
          check(cfdb_op_d2t(ctx, CFDB_F32, R, Uv->current_cu, Uv->prev_cu, dtv, Uv->has_prev ? 1 : 0, Uv->next_cu,
                            N),
                "cfdb_op_d2t");
        }
        std::swap(Uv->prev_cu, Uv->current_cu);  // prev <- current
        std::swap(Uv->current_cu, Uv->next_cu);  // current <- next
        Uv->has_prev = true;
      } else if (lhs->is_field) {
        const float* R = eval_node(rhs.node.get());
        check(cfdb_op_scalar(ctx, CFDB_F32, CFDB_OP_MUL, R, 1.0, lhs->next_cu, int64_t(lhs->mesh->_num_nodes)),
              "cfdb_op_scalar");
        std::swap(lhs->current_cu, lhs->next_cu);
      } else {
        throw std::runtime_error("Equation: left-hand side must be a field, d1t(field) or d2t(field)");
      }
    }
    // boundary functions in variable order; a run of consecutive boundary
    // copies on one mesh goes out as one launch (each writes only its own
    // field from its own buffer, so the run's order cannot matter)
    std::vector<void*> set_fields;
    std::vector<const void*> set_values;
    Mesh3D* set_mesh = nullptr;
    auto flush_sets = [&] {
      if (set_fields.empty()) return;
      check(cfdb_op_boundary_set_many(ctx, set_mesh->handle(), CFDB_F32, int32_t(set_fields.size()), set_fields.data(),
                                      set_values.data()),
            "cfdb_op_boundary_set_many");
      set_fields.clear();
      set_values.clear();
    };
    for (Variable* v : all_vars) {
      const BoundaryCopyCu* copy =
          v != bc_done && v->has_boundary_conditions_cu ? v->boundary_conditions_cu.target<BoundaryCopyCu>() : nullptr;
      if (copy && copy->count == v->mesh->_num_nodes) {
        if (set_mesh != v->mesh) flush_sets();
        set_mesh = v->mesh;
        set_fields.push_back(v->current_cu);
        set_values.push_back(copy->buf.get());
      } else {
        flush_sets();
      }
      if (copy && copy->count == v->mesh->_num_nodes) {
        // queued above
      } else if (v == bc_done) {
        // applied inside the fused step
      } else if (v->has_boundary_conditions_cu) {
        v->boundary_conditions_cu(v->mesh, v->current_cu, dt);
      } else if (v->boundary_conditions) {
        using Plain = HostVec (*)(Mesh3D*, HostVec&, const DT*);
        auto* f = v->boundary_conditions.target<Plain>();
        if (!(f && *f == &boundary_none)) {
          HostVec cur = v->host();
          v->set_current(v->boundary_conditions(v->mesh, cur, dt));
        }
      }
      bool store = !CFDArcoGlobalInit::skip_history;
      for (Variable* s : store_vars) store = store || (s == v && !CFDArcoGlobalInit::skip_history);
      if (store) {
        flush_sets();  // the stored state has its boundary copy
        v->history.push_back(v->host());
      }
    }
    flush_sets();
    if (visualize) std::printf("\rstep %zu / %zu", t + 1, timesteps);
  }
  check(cfdb_sync(ctx), "cfdb_sync");
  if (visualize) std::printf("\n");
  if (CFDArcoGlobalInit::jit_report) {
    const double ms_steps = ms_since(t_start) - ms_plan - ms_compile - ms_first;
    const auto t_free = Clock::now();
    units.clear();  // the plans' kernels and the scratch block, as the return would
    device_free(scratch.p);
    scratch.p = nullptr;
    std::fprintf(stderr,
                 "evaluate phases (ms): plan %.3f, kernel builds %.3f, first step %.3f, other steps %.3f, "
                 "release %.3f\n",
                 ms_plan, ms_compile, ms_first, ms_steps, ms_since(t_free));
  }
}

// ---------------------------------------------------------------------------
// output files (include/io_operators_tmpl.hpp)
// ---------------------------------------------------------------------------
namespace {
namespace fs = std::filesystem;

std::string var_dir(const Variable* v) {
  fs::path d = fs::path(CFDArcoGlobalInit::store_dir) / (v->name.empty() ? std::string("var") : v->name);
  fs::create_directories(d);
  return d.string();
}

void link_latest(const fs::path& latest) {
  std::error_code ec;
  fs::remove_all(latest, ec);
  fs::create_directory_symlink(fs::absolute(CFDArcoGlobalInit::store_dir), latest, ec);
  if (ec) throw std::runtime_error("run_latest link: " + ec.message());
}
}  // namespace

void store_history(const std::vector<Variable*>& vars_to_store, const Mesh3D* mesh) {
  if (CFDArcoGlobalInit::store_dir.empty()) throw std::runtime_error("store_history: call CFDArcoGlobalInit::initialize first");
  fs::create_directories(CFDArcoGlobalInit::store_dir);
  for (const Variable* v : vars_to_store) {
    const std::string dir = var_dir(v);
    // every stored entry but the last, as the reference (io_operators_tmpl.hpp:53)
    for (size_t i = 0; i + 1 < v->history.size(); ++i) {
      const std::string path = (fs::path(dir) / ("res_" + std::to_string(i) + ".vti")).string();
      check(cfdb_write_vti(path.c_str(), v->name.c_str(), int64_t(mesh->_x), int64_t(mesh->_y), int64_t(mesh->_z),
                           v->history[i].data()),
            "cfdb_write_vti");
    }
  }
  link_latest(fs::absolute(fs::path(CFDArcoGlobalInit::store_dir) / ".." / "run_latest"));
}

void init_store_history_stepping(const std::vector<Variable*>& vars_to_store, const Mesh3D* mesh,
                                 const std::string&) {
  if (CFDArcoGlobalInit::store_dir.empty())
    throw std::runtime_error("init_store_history_stepping: call CFDArcoGlobalInit::initialize first");
  CFDArcoGlobalInit::store_stepping = true;
  fs::create_directories(CFDArcoGlobalInit::store_dir);
  for (const Variable* v : vars_to_store) var_dir(v);
  store_mesh(mesh, CFDArcoGlobalInit::store_dir);
}

void store_history_stepping(const std::vector<Variable*>& vars_to_store, const Mesh3D*, int i) {
  for (Variable* v : vars_to_store) {
    const HostVec cur = v->host();
    const std::string path = (fs::path(var_dir(v)) / (std::to_string(i) + ".bin")).string();
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("store_history_stepping: cannot open " + path);
    const size_t w = std::fwrite(cur.data(), sizeof(float), cur.size(), f);
    const bool ok = std::fclose(f) == 0 && w == cur.size();
    if (!ok) throw std::runtime_error("store_history_stepping: writing " + path + " failed");
  }
}

void finalize_history_stepping(const std::string& store_path) {
  link_latest(fs::absolute(fs::path(store_path) / "run_latest"));
}

void store_mesh(const Mesh3D* mesh, const std::string& store_path) {
  fs::create_directories(store_path);
  const std::string path = (fs::path(store_path) / "mesh.json").string();
  check(cfdb_write_mesh_json(path.c_str(), int64_t(mesh->_x), int64_t(mesh->_y), int64_t(mesh->_z), mesh->_dx,
                             mesh->_dy, mesh->_dz, nullptr),
        "cfdb_write_mesh_json");
}

}  // namespace cfdb
