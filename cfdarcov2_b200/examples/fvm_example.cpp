// Drop-in usage of the C++ facade, written the way the reference's examples
// are (examples/main_3d_heat.cpp, examples/main_3d_wave.cu): a Mesh3D, field
// Variables with boundary functions, a DT policy, an EquationTemplate and
// Equation::evaluate.  The final fields are written as raw float32 to argv[2].
//
//   fvm_example heat     out.bin nx ny nz steps   d1t(T) = 0.01 lapl(T), zero-gradient walls (fused step)
//   fvm_example heat_bc  out.bin nx ny nz steps   same with the reference's boundary_copy_cu
//   fvm_example wave_d2t out.bin nx ny nz steps   d2t(u) = c^2 (d2dx(u) + d2dy(u)) (operator tree)
//   fvm_example advect   out.bin nx ny nz steps   q = q - dt (u d1dx(q) + v d1dy(q)) + 0.01 stab_tot(q),
//                                                 then d1t(r) = -d1dz(q) - r (operator tree)
//   fvm_example <mode>_nojit ...                  the same with use_jit = false: operator by operator
//                                                 instead of one generated kernel per equation
//   fvm_example nested   out.bin nx ny nz steps   d1t(q) = 0.01 lapl(d1dx(q) + q) - 0.001 stab_tot(d1dy(q))
//                                                 + d1dz(q q): operators of operators
//   fvm_example euler3d  out.bin nx ny nz steps   the reference's 20-equation Euler system (main_3d.cpp)
//   fvm_example ref_heat out.bin nx ny nz steps   the reference's heat benchmark (main_3d_heat.cpp)
//   fvm_example ref_wave out.bin nx ny nz steps   the reference's wave benchmark (main_3d_wave.cu)
//   fvm_example <mode>_twice ...                  evaluate twice, print evaluate_us and steady_us
//   fvm_example <mode>_arrays ...                 generated kernels read the face arrays on exact lattices too
//   fvm_example <mode>_report ...                 print each generated kernel's registers and local bytes
//   fvm_example heat_store out.bin nx ny nz steps dir
//                                                 heat with history kept, then the reference's output
//                                                 calls: store_history (.vti per step), mesh.json and
//                                                 one stepping .bin of the final state under dir
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "cfdb/fvm3d.hpp"

using namespace cfdb;

static int g_lattice = 0;  // lattice_equations of the last evaluate
static int g_groups = 0;   // jit_groups of the last evaluate

// Equation(steps).evaluate timed on the wall clock around the call, as the
// reference's examples time it (examples/main_3d.cpp: the time includes
// building the generated kernels): evaluate_us.  With `twice` a second call
// follows (kernels already built, the state advanced further): steady_us.
static int timed_evaluate(size_t steps, std::vector<Variable*>& vars, EquationTemplate& eqs, DT& dt, bool twice,
                          int* fused = nullptr) {
  auto run = [&](int* jitted) {
    const auto t0 = std::chrono::steady_clock::now();
    Equation eq(steps);
    eq.evaluate(vars, eqs, &dt, false);
    if (jitted) *jitted = eq.jit_equations;
    if (fused) *fused = eq.fused_equations;
    g_lattice = eq.lattice_equations;
    g_groups = eq.jit_groups;
    return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
  };
  int jitted = 0;
  std::printf("evaluate_us=%.0f\n", run(&jitted));
  if (twice) std::printf("steady_us=%.0f\n", run(nullptr));
  return jitted;
}

static HostVec gaussian(Mesh3D& m, float cx, float cy, float cz, float sigma) {
  HostVec v(m._num_nodes);
  for (size_t i = 0; i < m._num_nodes; ++i) {
    const float dx = m.x(i) - cx, dy = m.y(i) - cy, dz = m.z(i) - cz;
    v[i] = std::exp(-(dx * dx + dy * dy + dz * dz) / (2 * sigma * sigma));
  }
  return v;
}

int main(int argc, char** argv) {
  if (argc < 7) {
    std::fprintf(stderr, "usage: %s mode out.bin nx ny nz steps\n", argv[0]);
    return 2;
  }
  // "<mode>_twice": evaluate twice (second timing without kernel builds);
  // "<mode>_nojit": the same equations with use_jit = false (operator-by-operator path);
  // "<mode>_arrays": generated kernels read the face arrays even on an exact lattice
  std::string mode = argv[1];
  auto suffix = [&](const char* s) {
    const size_t k = std::strlen(s);
    if (mode.size() <= k || mode.compare(mode.size() - k, k, s) != 0) return false;
    mode.resize(mode.size() - k);
    return true;
  };
  const bool report = suffix("_report");
  const bool twice = suffix("_twice");
  const bool arrays = suffix("_arrays");
  const bool jit = !suffix("_nojit");
  const char* out = argv[2];
  const size_t nx = std::strtoul(argv[3], nullptr, 10), ny = std::strtoul(argv[4], nullptr, 10),
               nz = std::strtoul(argv[5], nullptr, 10);
  const size_t steps = std::strtoul(argv[6], nullptr, 10);
  try {
    const bool storing = mode == "heat_store";
    if (storing && argc < 8) {
      std::fprintf(stderr, "heat_store needs a store directory\n");
      return 2;
    }
    CFDArcoGlobalInit::initialize(argc, argv, !storing, storing ? argv[7] : "./dumps");
    CFDArcoGlobalInit::enable_cuda(0);
    CFDArcoGlobalInit::jit_lattice = !arrays;
    CFDArcoGlobalInit::jit_all = jit;
    CFDArcoGlobalInit::jit_report = report;
    Mesh3D mesh(nx, ny, nz, 1.f / float(nx), 1.f / float(ny), 1.f / float(nz));
    mesh.init_basic_internals();
    mesh.compute();
    std::vector<HostVec> result;
    int fused = 0, jitted = 0;
    const auto t0 = std::chrono::steady_clock::now();
    if (mode == "heat" || mode == "heat_bc" || storing) {
      HostVec T0 = gaussian(mesh, 0.5f, 0.5f, 0.5f, 0.1f);
      Variable T = mode == "heat_bc" ? Variable(&mesh, T0, boundary_none, boundary_copy_cu(&mesh, T0), "T")
                                     : Variable(&mesh, T0, boundary_none, "T");
      std::vector<Variable*> space_vars{&T};
      const float h = 1.f / float(nx);
      DT dt(&mesh, UpdatePolicies::constant_dt, 0.1f * h * h / 0.01f, space_vars);
      EquationTemplate eqs = {{d1t(T), '=', 0.01f * lapl(T), jit}};
      Equation eq(steps);
      eq.evaluate(space_vars, eqs, &dt, false, {&T});
      fused = eq.fused_equations;
      jitted = eq.jit_equations;
      g_lattice = eq.lattice_equations;
      g_groups = eq.jit_groups;
      result.push_back(T.host());
      if (storing) {
        store_history({&T}, &mesh);
        init_store_history_stepping({&T}, &mesh, argv[7]);
        store_history_stepping({&T}, &mesh, int(steps));
        finalize_history_stepping(argv[7]);
      }
    } else if (mode == "wave_d2t") {
      HostVec U0 = gaussian(mesh, 0.5f, 0.5f, 0.5f, 0.15f);
      Variable u(&mesh, U0, boundary_none, "u");
      std::vector<Variable*> vars{&u};
      const float c = 0.3f;
      DT dt(&mesh, UpdatePolicies::constant_dt, 0.01f, vars);
      EquationTemplate eqs = {{d2t(u), '=', c * c * (d2dx(u) + d2dy(u)), jit}};
      Equation eq(steps);
      eq.evaluate(vars, eqs, &dt, false);
      jitted = eq.jit_equations;
      fused = eq.fused_equations;
      g_lattice = eq.lattice_equations;
      g_groups = eq.jit_groups;
      result.push_back(u.host());
    } else if (mode == "advect") {
      HostVec Q0 = gaussian(mesh, 0.4f, 0.5f, 0.5f, 0.15f), Uv(mesh._num_nodes, 0.3f), Vv(mesh._num_nodes, -0.2f),
              R0(mesh._num_nodes, 0.f);
      Variable q(&mesh, Q0, boundary_none, "q"), u(&mesh, Uv, boundary_none, "u"), v(&mesh, Vv, boundary_none, "v"),
          r(&mesh, R0, boundary_none, "r");
      std::vector<Variable*> vars{&q, &u, &v, &r};
      DT dt(&mesh, UpdatePolicies::constant_dt, 0.002f, vars);
      EquationTemplate eqs = {
          {&q, '=', q - dt * (u * d1dx(q) + v * d1dy(q)) + 0.01f * stab_tot(q), jit},
          {d1t(r), '=', -d1dz(q) - r, jit},
      };
      Equation eq(steps);
      eq.evaluate(vars, eqs, &dt, false);
      jitted = eq.jit_equations;
      g_lattice = eq.lattice_equations;
      g_groups = eq.jit_groups;
      result.push_back(q.host());
      result.push_back(r.host());
    } else if (mode == "nested") {
      // operators of operators: the generated plan materialises d1dx(q) + q and
      // d1dy(q) in passes of their own before the outer lapl / stab_tot
      HostVec Q0 = gaussian(mesh, 0.5f, 0.45f, 0.55f, 0.15f);
      Variable q(&mesh, Q0, boundary_none, "q");
      std::vector<Variable*> vars{&q};
      DT dt(&mesh, UpdatePolicies::constant_dt, 0.001f, vars);
      EquationTemplate eqs = {
          {d1t(q), '=', 0.01f * lapl(d1dx(q) + q) - 0.001f * stab_tot(d1dy(q)) + d1dz(q * q), jit},
      };
      Equation eq(steps);
      eq.evaluate(vars, eqs, &dt, false);
      jitted = eq.jit_equations;
      g_lattice = eq.lattice_equations;
      g_groups = eq.jit_groups;
      result.push_back(q.host());
    } else if (mode == "euler3d") {
      // The reference's "euler" benchmark system (examples/main_3d.cpp): primitive
      // and conservative variables, 15 use_jit equations (primitive recovery,
      // a half-step predictor, conservative fluxes) and 5 operator-path
      // updates with stab_tot dissipation; gamma 5/3, CFL time step, Dirichlet
      // boundary layers holding the initial values.  The reference's mesh
      // defaults: unit cells (dx = dy = dz = 1, so V = 1: the scheme adds
      // per-volume fluxes to per-cell conservative variables), CFL 0.005
      // (include/utils3d.hpp:35-66).
      Mesh3D cube(nx, ny, nz, 1.f, 1.f, 1.f);
      cube.init_basic_internals();
      cube.compute();
      Mesh3D& mesh = cube;  // this system runs on the unit-cell mesh
      const size_t N = mesh._num_nodes;
      HostVec r0(N), u0(N), v0(N), w0(N, 0.6f), p0(N, 2.5f), vol(N, mesh._dx * mesh._dy * mesh._dz);
      for (size_t i = 0; i < N; ++i) {
        const float x = mesh.x(i), y = mesh.y(i), z = mesh.z(i);
        const bool jet = 0.4f * mesh._lx < x && x < 0.6f * mesh._lx && 0.4f * mesh._ly < y && y < 0.6f * mesh._ly;
        r0[i] = jet ? 5.f : 1.f;
        const int band = int(z / (0.1f * mesh._lz));  // alternating shear bands in z
        u0[i] = v0[i] = (band % 2 == 0) ? -0.1f : 0.1f;
      }
      const float gamma = 5.f / 3.f;
      HostVec m0(N), mu0(N), mv0(N), mw0(N), e0(N);
      for (size_t i = 0; i < N; ++i) {
        m0[i] = r0[i] * vol[i];
        mu0[i] = r0[i] * u0[i] * vol[i];
        mv0[i] = r0[i] * v0[i] * vol[i];
        mw0[i] = r0[i] * w0[i] * vol[i];
        e0[i] = (p0[i] / (gamma - 1) + 0.5f * r0[i] * (u0[i] * u0[i] + v0[i] * v0[i] + w0[i] * w0[i])) * vol[i];
      }
      auto fixed = [&](HostVec& init, const char* name) {
        return Variable(&mesh, init, boundary_none, boundary_copy_cu(&mesh, init), name);
      };
      Variable rho = fixed(r0, "rho"), u = fixed(u0, "u"), v = fixed(v0, "v"), w = fixed(w0, "w"), p = fixed(p0, "p");
      Variable mass = fixed(m0, "mass"), rho_u = fixed(mu0, "rho_u"), rho_v = fixed(mv0, "rho_v"),
               rho_w = fixed(mw0, "rho_w"), rho_e = fixed(e0, "rho_e");
      Variable mass_tmp(&mesh, m0, boundary_none, "mass_tmp"), rho_u_tmp(&mesh, mu0, boundary_none, "rho_u_tmp"),
          rho_v_tmp(&mesh, mv0, boundary_none, "rho_v_tmp"), rho_w_tmp(&mesh, mw0, boundary_none, "rho_w_tmp"),
          rho_e_tmp(&mesh, e0, boundary_none, "rho_e_tmp"), volumes(&mesh, vol, boundary_none, "volumes");
      Variable E = p / (gamma - 1) + 0.5f * rho * ((u * u) + (v * v) + (w * w));
      std::vector<Variable*> space_vars{&u, &v, &w, &p, &rho};
      DT dt(&mesh, UpdatePolicies::CourantFriedrichsLewy3D, 0.005f, space_vars);
      const float dissip = 2.f;
      EquationTemplate eqs = {
          {&rho, '=', mass / volumes, jit},
          {&u, '=', rho_u / rho / volumes, jit},
          {&v, '=', rho_v / rho / volumes, jit},
          {&w, '=', rho_w / rho / volumes, jit},
          {&p, '=', (rho_e / volumes - 0.5f * rho * (u * u + v * v + w * w)) * (gamma - 1), jit},
          {&rho, '=', rho - 0.5f * dt * (u * d1dx(rho) + rho * d1dx(u) + v * d1dy(rho) + rho * d1dy(v) +
                                         w * d1dz(rho) + rho * d1dz(w)), jit},
          {&u, '=', u - 0.5f * dt * (u * d1dx(u) + v * d1dy(u) + w * d1dz(u) + (1.f / rho) * d1dx(p)), jit},
          {&v, '=', v - 0.5f * dt * (u * d1dx(v) + v * d1dy(v) + w * d1dz(v) + (1.f / rho) * d1dy(p)), jit},
          {&w, '=', w - 0.5f * dt * (u * d1dx(w) + v * d1dy(w) + w * d1dz(w) + (1.f / rho) * d1dz(p)), jit},
          {&p, '=', p - 0.5f * dt * (gamma * p * (d1dx(u) + d1dy(v) + d1dz(w)) + u * d1dx(p) + v * d1dy(p) +
                                     w * d1dz(p)), jit},
          {&mass_tmp, '=', 0.f * mass_tmp - (d1dx(rho * u) + d1dy(rho * v) + d1dz(rho * w)), jit},
          {&rho_u_tmp, '=', 0.f * rho_u_tmp - (d1dx(rho * u * u + p) + d1dy(rho * v * u) + d1dz(rho * w * u)), jit},
          {&rho_v_tmp, '=', 0.f * rho_v_tmp - (d1dx(rho * v * u) + d1dy(rho * v * v + p) + d1dz(rho * v * w)), jit},
          {&rho_w_tmp, '=', 0.f * rho_w_tmp - (d1dx(rho * w * u) + d1dy(rho * w * v) + d1dz(rho * w * w + p)), jit},
          {&rho_e_tmp, '=', 0.f * rho_e_tmp - (d1dx((E + p) * u) + d1dy((E + p) * v) + d1dz((E + p) * w)), jit},
          {d1t(mass), '=', mass_tmp - stab_tot(rho) * dissip, false},
          {d1t(rho_u), '=', rho_u_tmp - stab_tot(rho * u) * dissip, false},
          {d1t(rho_v), '=', rho_v_tmp - stab_tot(rho * v) * dissip, false},
          {d1t(rho_w), '=', rho_w_tmp - stab_tot(rho * w) * dissip, false},
          {d1t(rho_e), '=', rho_e_tmp - stab_tot(E) * dissip, false},
      };
      std::vector<Variable*> all_vars{&rho, &u, &v, &w, &p, &mass, &rho_u, &rho_v, &rho_w, &rho_e};
      jitted = timed_evaluate(steps, all_vars, eqs, dt, twice);
      for (Variable* x : {&rho, &u, &v, &w, &p}) result.push_back(x->host());
    } else if (mode == "ref_heat") {
      // the reference's heat benchmark (examples/main_3d_heat.cpp): unit cells, T = 100
      // in the two lowest z layers, boundary copy, dt 0.005, d1t(T) = 3 lapl(T)
      Mesh3D cube(nx, ny, nz, 1.f, 1.f, 1.f);
      cube.init_basic_internals();
      cube.compute();
      HostVec T0(cube._num_nodes);
      for (size_t i = 0; i < cube._num_nodes; ++i) T0[i] = cube.z(i) < 2.f * cube._dz ? 100.f : 0.f;
      Variable T(&cube, T0, boundary_none, boundary_copy_cu(&cube, T0), "T");
      std::vector<Variable*> vars{&T};
      DT dt(&cube, UpdatePolicies::constant_dt, 0.005f, vars);
      EquationTemplate eqs = {{d1t(T), '=', 3.0f * lapl(T), jit}};
      jitted = timed_evaluate(steps, vars, eqs, dt, twice, &fused);
      result.push_back(T.host());
    } else if (mode == "ref_wave") {
      // the reference's wave benchmark (examples/main_3d_wave.cu): unit cells, u = 0,
      // sin(0.2 t) driven at the cells (0.1, 0.1, 0.1) and (0.9, 0.9, 0.9) of the box,
      // dt 0.1, c 0.3, d2t(u) = c^2 (d2dx(u) + d2dy(u)); the driver is applied on the
      // device (the reference's boundary_sine_cu) instead of through host memory
      Mesh3D cube(nx, ny, nz, 1.f, 1.f, 1.f);
      cube.init_basic_internals();
      cube.compute();
      HostVec U0(cube._num_nodes, 0.f);
      const size_t n1 = cube.square_node_coord_to_idx(size_t(nx * 0.1), size_t(ny * 0.1), size_t(nz * 0.1));
      const size_t n2 = cube.square_node_coord_to_idx(size_t(nx * 0.9), size_t(ny * 0.9), size_t(nz * 0.9));
      BoundaryFNCU sine = [n1, n2](Mesh3D*, float* field, const DT* d) {
        // sin of float(step) * 0.2 in double, stored as float (main_3d_wave.cu:33-42)
        const float s = float(std::sin(double(float(d->_current_time_step_int)) * 0.2));
        check(cfdb_op_fill(CFDArcoGlobalInit::ctx(), CFDB_F32, field + n1, s, 1), "cfdb_op_fill");
        check(cfdb_op_fill(CFDArcoGlobalInit::ctx(), CFDB_F32, field + n2, s, 1), "cfdb_op_fill");
      };
      Variable u(&cube, U0, boundary_none, sine, "u");
      std::vector<Variable*> vars{&u};
      DT dt(&cube, UpdatePolicies::constant_dt, 0.1f, vars);
      const float c = 0.3f;
      EquationTemplate eqs = {{d2t(u), '=', c * c * (d2dx(u) + d2dy(u)), jit}};
      jitted = timed_evaluate(steps, vars, eqs, dt, twice, &fused);
      result.push_back(u.host());
    } else {
      std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
      return 2;
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    FILE* f = std::fopen(out, "wb");
    if (!f) return 3;
    for (const auto& v : result) std::fwrite(v.data(), sizeof(float), v.size(), f);
    std::fclose(f);
    double sum = 0, mx = -1e30;
    for (float x : result[0]) {
      sum += x;
      mx = x > mx ? x : mx;
    }
    std::printf(
        "mode=%s cells=%zu steps=%zu fused_equations=%d jit_equations=%d lattice_equations=%d jit_groups=%d sum=%.9g "
        "max=%.9g seconds=%.6f\n",
        mode.c_str(), mesh._num_nodes, steps, fused, jitted, g_lattice, g_groups, sum, mx, secs);
    CFDArcoGlobalInit::finalize();
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
