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
  // "<mode>_nojit": the same equations with use_jit = false (operator-by-operator path)
  std::string mode = argv[1];
  const bool jit = mode.size() < 6 || mode.compare(mode.size() - 6, 6, "_nojit") != 0;
  if (!jit) mode.resize(mode.size() - 6);
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
      result.push_back(q.host());
      result.push_back(r.host());
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
    std::printf("mode=%s cells=%zu steps=%zu fused_equations=%d jit_equations=%d sum=%.9g max=%.9g seconds=%.6f\n",
                mode.c_str(), mesh._num_nodes, steps, fused, jitted, sum, mx, secs);
    CFDArcoGlobalInit::finalize();
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
