// Drop-in C++ facade of the reference's finite-volume DSL
// (include/fvm3d.hpp of int0vrt/cfdARCOV2): Variable expression trees with
// + - * /, d1dx..d1dz, d2dx..d2dz, lapl, stab*, d1t, d2t, DT, UpdatePolicies,
// EquationTemplate and Equation::evaluate.  Expressions are evaluated on the
// GPU through libcfdb's operator kernels into pooled device buffers (no
// allocation per step after the first); the heat template
//   {d1t(T), '=', k * lapl(T), ...}
// on a uniform mesh runs as the fused TMA step instead of an operator tree
// (the role of the reference's KernelBuilder, src/fvm3d.cpp:1219-1394).
//
// Semantics kept from the reference: equations run in order within a step
// and later ones see earlier updates (src/fvm3d.cpp:1012-1032); boundary
// functions run after all equations (src/fvm3d.cpp:1036-1049).  Deliberate
// differences: a plain Variable left-hand side is written to a fresh buffer
// and swapped in (Jacobi), not in place (the JIT race of src/fvm3d.cpp:53,81);
// the first d1t/d2t step starts from the initial state (the JIT's jit_post
// aliasing, src/fvm3d.cpp:993-996); d2t keeps its previous state on the
// device whether or not history is stored (src/fvm3d.cpp:735-740).
#pragma once

#include <functional>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "cfdb/mesh3d.hpp"

namespace cfdb {

class DT;
class Variable;
struct Node;

using HostVec = std::vector<float>;

// Host boundary function: new host values from the current ones
// (BoundaryFN, include/fvm3d.hpp:40).
using BoundaryFN = std::function<HostVec(Mesh3D*, HostVec&, const DT*)>;
// Device boundary function: updates the device field in place
// (BoundaryFNCU, include/fvm3d.hpp:41).
using BoundaryFNCU = std::function<void(Mesh3D*, float* device_field, const DT*)>;

// _boundary_copy_cu of the reference examples (examples/main_3d_heat.cpp:41-60):
// boundary-layer cells are reset to `values`.
BoundaryFNCU boundary_copy_cu(Mesh3D* mesh, const HostVec& values);
HostVec boundary_none(Mesh3D*, HostVec& arr, const DT*);

class Variable {
 public:
  Variable();
  Variable(Mesh3D* mesh, HostVec& initial, BoundaryFN bc, std::string name = "");
  Variable(Mesh3D* mesh, HostVec& initial, BoundaryFN bc, BoundaryFNCU bc_cu, std::string name = "");
  Variable(Mesh3D* mesh, float value);
  virtual ~Variable();
  Variable(const Variable&) = default;
  Variable& operator=(const Variable&) = default;

  Variable operator+(const Variable& r) const;
  Variable operator-(const Variable& r) const;
  Variable operator*(const Variable& r) const;
  Variable operator/(const Variable& r) const;
  Variable operator-() const;

  // Host copy of the current state (synchronous).
  const HostVec& host();
  void set_current(const HostVec& values);
  const std::vector<HostVec>& get_history() const { return history; }

  std::string name;
  Mesh3D* mesh = nullptr;
  HostVec current;  // host mirror, refreshed by host()
  std::vector<HostVec> history;
  std::shared_ptr<Node> node;

  // device state of a field variable
  float* current_cu = nullptr;
  float* next_cu = nullptr;
  float* prev_cu = nullptr;  // d2t only
  bool has_prev = false;
  BoundaryFN boundary_conditions;
  BoundaryFNCU boundary_conditions_cu;
  bool has_boundary_conditions_cu = false;
  bool is_field = false;
};

Variable operator+(float l, const Variable& r);
Variable operator-(float l, const Variable& r);
Variable operator*(float l, const Variable& r);
Variable operator/(float l, const Variable& r);
Variable operator+(const Variable& l, float r);
Variable operator-(const Variable& l, float r);
Variable operator*(const Variable& l, float r);
Variable operator/(const Variable& l, float r);

// Time-derivative left-hand sides (DtVar / D2tVar, include/fvm3d.hpp:250-318).
class DtVar : public Variable {
 public:
  explicit DtVar(Variable* v) : var(v) {}
  Variable* var;
};
class D2tVar : public Variable {
 public:
  explicit D2tVar(Variable* v) : var(v) {}
  Variable* var;
};

DtVar* d1t(Variable& v);
D2tVar* d2t(Variable& v);

Variable d1dx(const Variable& v);
Variable d1dy(const Variable& v);
Variable d1dz(const Variable& v);
Variable d2dx(const Variable& v);
Variable d2dy(const Variable& v);
Variable d2dz(const Variable& v);
Variable lapl(const Variable& v);
Variable stab_tot(const Variable& v);
Variable stabx(const Variable& v);
Variable staby(const Variable& v);
Variable stabz(const Variable& v);

// Time step (DT, include/fvm3d.hpp:209-248).  update_fn returns dt from
// (CFL, space variables, mesh); space variables are read on the device.
class DT : public Variable {
 public:
  using UpdateFn = std::function<float(float, std::vector<Variable*>&, Mesh3D*)>;
  DT(Mesh3D* mesh, UpdateFn update_fn, float CFL, std::vector<Variable*> space_vars = {});
  void update();
  UpdateFn update_fn;
  float CFL;
  std::vector<Variable*> space_vars;
  float _dt = 0.f;
  size_t _current_time_step_int = 0;
  double _current_time_dbl = 0.0;
};

// UpdatePolicies (src/fvm3d.cpp:497-567); the CFL policies evaluate on the
// device (cfdb_cfl_dt) with gamma = 5/3 as the reference hard-codes.
struct UpdatePolicies {
  static float constant_dt(float CFL, std::vector<Variable*>&, Mesh3D*) { return CFL; }
  static float CourantFriedrichsLewy3D(float CFL, std::vector<Variable*>& vars, Mesh3D* mesh);  // u, v, w, p, rho
  static float CourantFriedrichsLewy1D(float CFL, std::vector<Variable*>& vars, Mesh3D* mesh);  // u, p, rho
};

using EquationTemplate = std::vector<std::tuple<Variable*, char, Variable, bool>>;

class Equation {
 public:
  explicit Equation(size_t timesteps);
  void evaluate(std::vector<Variable*>& all_vars, EquationTemplate& equation_system, DT* dt, bool visualize,
                std::vector<Variable*> store_vars = {}) const;
  size_t timesteps;
  // number of equations the last evaluate() ran as hand-written fused kernels
  mutable int fused_equations = 0;
  // number of use_jit equations the last evaluate() ran as one generated,
  // run-time compiled kernel each (KernelBuilder, src/fvm3d.cpp:1219-1394)
  mutable int jit_equations = 0;
  // of those, the equations whose kernels take an exact lattice's geometry as constants
  mutable int lattice_equations = 0;
  // kernels the generated plain / d1t equations fuse into (one per group of consecutive equations)
  mutable int jit_groups = 0;
};

// Output of the reference's include/io_operators_tmpl.hpp, written through
// libcfdb's headless writers (no VTK, no nlohmann::json):
//   store_history            store_dir/<name>/res_<i>.vti for each stored history entry but the
//                            last, then store_dir/../run_latest -> store_dir (lines 44-103)
//   init_store_history_stepping  directories + mesh.json (lines 105-120)
//   store_history_stepping   store_dir/<name>/<i>.bin, raw float32 in cell order (lines 133-159)
//   finalize_history_stepping    store_path/run_latest -> store_dir (lines 121-128)
//   store_mesh               store_path/mesh.json (lines 161-212)
void store_history(const std::vector<Variable*>& vars_to_store, const Mesh3D* mesh);
void init_store_history_stepping(const std::vector<Variable*>& vars_to_store, const Mesh3D* mesh,
                                 const std::string& store_path = "./dumps");
void store_history_stepping(const std::vector<Variable*>& vars_to_store, const Mesh3D* mesh, int i);
void finalize_history_stepping(const std::string& store_path = "./dumps");
void store_mesh(const Mesh3D* mesh, const std::string& store_path);

}  // namespace cfdb
