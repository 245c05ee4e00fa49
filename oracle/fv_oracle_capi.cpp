// fv_oracle_capi.cpp -- TEST INFRASTRUCTURE ONLY.
// extern "C" wrappers over fv_oracle.hpp so that the tests, the smoke check
// and the CPU-baseline leg of bench.py can drive the restatement through
// ctypes.  Every function exists in an _f64 and an _f32 flavour.  Parity
// status: unpinned (see fv_oracle.hpp).
#include "fv_oracle.hpp"

#include <chrono>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace fvo;

namespace {

template <class R> Mesh<R>* M(void* h) { return static_cast<Mesh<R>*>(h); }

template <class R>
void export_mesh(const Mesh<R>& m, R* normal, R* normal_alt, R* area, R* alpha, R* len, R* vol, R* center,
                 R* isb, int64_t* ids, int64_t* ibf) {
  const int64_t n = m.n;
  for (int d = 0; d < 3; ++d) {
    if (normal) std::memcpy(normal + d * 6 * n, m.normal[d].data(), sizeof(R) * 6 * n);
    if (normal_alt) std::memcpy(normal_alt + d * 6 * n, m.normal_alt[d].data(), sizeof(R) * 6 * n);
    if (center) std::memcpy(center + d * n, m.center[d].data(), sizeof(R) * n);
  }
  if (area) std::memcpy(area, m.area.data(), sizeof(R) * 6 * n);
  if (alpha) std::memcpy(alpha, m.alpha_d.data(), sizeof(R) * 6 * n);
  if (len) std::memcpy(len, m.len_c2f.data(), sizeof(R) * 6 * n);
  if (vol) std::memcpy(vol, m.volume.data(), sizeof(R) * n);
  if (isb) std::memcpy(isb, m.is_boundary.data(), sizeof(R) * n);
  if (ids) std::memcpy(ids, m.ids.data(), sizeof(int64_t) * 6 * n);
  if (ibf) std::memcpy(ibf, m.ids_bound_free.data(), sizeof(int64_t) * 6 * n);
}

template <class R> void heat_solve(const Mesh<R>& m, R* T, R k, R dt, int steps, int faithful) {
  std::vector<R> a(T, T + m.n), b(m.n), tmp;
  for (int s = 0; s < steps; ++s) {
    if (faithful) heat_step_faithful(m, a.data(), b.data(), k, dt, tmp);
    else heat_step(m, a.data(), b.data(), k, dt);
    a.swap(b);
  }
  std::memcpy(T, a.data(), sizeof(R) * m.n);
}

template <class R>
void wave_solve(const Mesh<R>& m, R* q, const R* c, R cconst, int mode, R dt, int steps, int faithful) {
  std::vector<R> a(q, q + 4 * m.n), b(4 * m.n), tmp;
  for (int s = 0; s < steps; ++s) {
    if (faithful && !c && mode == 0) wave_step_faithful(m, a.data(), b.data(), cconst, dt, tmp);
    else wave_step(m, a.data(), b.data(), c, cconst, mode, dt);
    a.swap(b);
  }
  std::memcpy(q, a.data(), sizeof(R) * 4 * m.n);
}

// Forward run that keeps every state (for the adjoint), J = 0.5 |p_T - target|^2,
// then the reverse sweep.  grad_c and grad_p0 are outputs (n values each).
template <class R>
double wave_gradient(const Mesh<R>& m, const R* q0, const R* c, const R* target, R dt, int steps, R* grad_c,
                     R* grad_p0) {
  const int64_t n = m.n;
  std::vector<R> states(size_t(steps + 1) * 4 * n);
  std::memcpy(states.data(), q0, sizeof(R) * 4 * n);
  for (int s = 0; s < steps; ++s)
    wave_step(m, states.data() + size_t(s) * 4 * n, states.data() + size_t(s + 1) * 4 * n, c, R(0), 1, dt);
  const R* qT = states.data() + size_t(steps) * 4 * n;
  double J = 0;
  std::vector<R> lam(4 * n, R(0)), lam0(4 * n);
  for (int64_t i = 0; i < n; ++i) {
    R d = qT[i] - target[i];
    J += 0.5 * double(d) * double(d);
    lam[i] = d;
  }
  for (int64_t i = 0; i < n; ++i) grad_c[i] = 0;
  for (int s = steps - 1; s >= 0; --s) {
    wave_adjoint_step(m, states.data() + size_t(s) * 4 * n, lam.data(), lam0.data(), c, grad_c, dt);
    lam.swap(lam0);
  }
  for (int64_t i = 0; i < n; ++i) grad_p0[i] = lam[i];
  return J;
}

template <class R> double wave_objective(const Mesh<R>& m, const R* q0, const R* c, const R* target, R dt, int steps) {
  const int64_t n = m.n;
  std::vector<R> a(q0, q0 + 4 * n), b(4 * n);
  for (int s = 0; s < steps; ++s) {
    wave_step(m, a.data(), b.data(), c, R(0), 1, dt);
    a.swap(b);
  }
  double J = 0;
  for (int64_t i = 0; i < n; ++i) {
    double d = double(a[i]) - double(target[i]);
    J += 0.5 * d * d;
  }
  return J;
}

// Euler to t_end: dt = cfl / (lam_x/dx + lam_y/dy + lam_z/dz), the last step
// clipped onto t_end; totals[2s], totals[2s+1] = sum rho V, sum E V after step
// s (s = 0 is the initial state).
template <class R>
int euler_solve(const Mesh<R>& m, R* U, R gamma, double cfl, double t_end, int max_steps, double* t_out,
                double* totals) {
  const int64_t n = m.n;
  std::vector<R> a(U, U + 5 * n), b(5 * n);
  double t = 0;
  int s = 0;
  if (totals) { totals[0] = neumaier_total(m, a.data()); totals[1] = neumaier_total(m, a.data() + 4 * n); }
  while (t < t_end && s < max_steps) {
    R lam[3];
    euler_max_speeds(m, a.data(), gamma, lam);
    double rate = (double(lam[0]) / double(m.dx) + double(lam[1]) / double(m.dy)) + double(lam[2]) / double(m.dz);
    double dt = cfl / rate;
    bool last = false;
    if (dt >= t_end - t) { dt = t_end - t; last = true; }
    euler_step(m, a.data(), b.data(), gamma, R(dt));
    a.swap(b);
    t = last ? t_end : t + dt;
    ++s;
    if (totals) {
      totals[2 * s] = neumaier_total(m, a.data());
      totals[2 * s + 1] = neumaier_total(m, a.data() + 4 * n);
    }
  }
  std::memcpy(U, a.data(), sizeof(R) * 5 * n);
  if (t_out) *t_out = t;
  return s;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

#define FVO_EXPORTS(SUF, R)                                                                                     \
  extern "C" void* fvo_mesh_create_##SUF(int64_t nx, int64_t ny, int64_t nz, double dx, double dy, double dz,   \
                                         const double* verts, int mode) {                                    \
    auto* m = new Mesh<R>();                                                                                   \
    build_mesh(*m, nx, ny, nz, dx, dy, dz, verts, mode);                                                     \
    return m;                                                                                                  \
  }                                                                                                            \
  extern "C" void fvo_mesh_destroy_##SUF(void* h) { delete M<R>(h); }                                          \
  extern "C" void fvo_mesh_export_##SUF(void* h, R* nrm, R* nalt, R* area, R* alpha, R* len, R* vol, R* ctr,   \
                                        R* isb, int64_t* ids, int64_t* ibf) {                                  \
    export_mesh(*M<R>(h), nrm, nalt, area, alpha, len, vol, ctr, isb, ids, ibf);                               \
  }                                                                                                            \
  extern "C" void fvo_grad_##SUF(void* h, const R* phi, R* out, int mask) { op_grad(*M<R>(h), phi, out, mask); } \
  extern "C" void fvo_lapl_##SUF(void* h, const R* phi, R* out, int mask) { op_lapl(*M<R>(h), phi, out, mask); } \
  extern "C" void fvo_stab_##SUF(void* h, const R* phi, R* out, int mask) { op_stab(*M<R>(h), phi, out, mask); } \
  extern "C" double fvo_cfl_reference_##SUF(void* h, double cfl, double gamma, const R* p, const R* rho,       \
                                            const R* u, const R* v, const R* w) {                              \
    return double(cfl_reference(*M<R>(h), R(cfl), R(gamma), p, rho, u, v, w));                                 \
  }                                                                                                            \
  extern "C" void fvo_heat_solve_##SUF(void* h, R* T, double k, double dt, int steps, int faithful) {          \
    heat_solve(*M<R>(h), T, R(k), R(dt), steps, faithful);                                                     \
  }                                                                                                            \
  extern "C" double fvo_heat_time_##SUF(void* h, R* T, double k, double dt, int steps, int faithful) {         \
    double t0 = now_s();                                                                                       \
    heat_solve(*M<R>(h), T, R(k), R(dt), steps, faithful);                                                     \
    return now_s() - t0;                                                                                       \
  }                                                                                                            \
  extern "C" void fvo_wave_rhs_##SUF(void* h, const R* q, const R* c, double cconst, int mode, R* out) {       \
    const Mesh<R>& m = *M<R>(h);                                                                               \
    for (int64_t i = 0; i < m.n; ++i) {                                                                        \
      R r[4];                                                                                                  \
      wave_rhs_cell(m, q, c, R(cconst), mode, i, r);                                                           \
      for (int k = 0; k < 4; ++k) out[k * m.n + i] = r[k];                                                     \
    }                                                                                                          \
  }                                                                                                            \
  extern "C" void fvo_wave_solve_##SUF(void* h, R* q, const R* c, double cconst, int mode, double dt,          \
                                       int steps, int faithful) {                                              \
    wave_solve(*M<R>(h), q, c, R(cconst), mode, R(dt), steps, faithful);                                       \
  }                                                                                                            \
  extern "C" double fvo_wave_time_##SUF(void* h, R* q, double cconst, double dt, int steps, int faithful) {    \
    double t0 = now_s();                                                                                       \
    wave_solve(*M<R>(h), q, (const R*)nullptr, R(cconst), 0, R(dt), steps, faithful);                          \
    return now_s() - t0;                                                                                       \
  }                                                                                                            \
  extern "C" double fvo_wave_dt_##SUF(void* h, const R* c, double cconst, double cfl) {                        \
    return wave_dt(*M<R>(h), c, cconst, cfl);                                                                  \
  }                                                                                                            \
  extern "C" void fvo_wave_adjoint_step_##SUF(void* h, const R* q, const R* lam1, R* lam0, const R* c, R* gc,  \
                                              double dt) {                                                     \
    wave_adjoint_step(*M<R>(h), q, lam1, lam0, c, gc, R(dt));                                                  \
  }                                                                                                            \
  extern "C" double fvo_wave_gradient_##SUF(void* h, const R* q0, const R* c, const R* target, double dt,      \
                                            int steps, R* gc, R* gp0) {                                        \
    return wave_gradient(*M<R>(h), q0, c, target, R(dt), steps, gc, gp0);                                      \
  }                                                                                                            \
  extern "C" double fvo_wave_objective_##SUF(void* h, const R* q0, const R* c, const R* target, double dt,     \
                                             int steps) {                                                      \
    return wave_objective(*M<R>(h), q0, c, target, R(dt), steps);                                              \
  }                                                                                                            \
  extern "C" void fvo_euler_rhs_##SUF(void* h, const R* U, double gamma, R* out) {                             \
    const Mesh<R>& m = *M<R>(h);                                                                               \
    for (int64_t i = 0; i < m.n; ++i) {                                                                        \
      R r[5];                                                                                                  \
      euler_rhs_cell(m, U, R(gamma), i, r);                                                                    \
      for (int k = 0; k < 5; ++k) out[k * m.n + i] = r[k];                                                     \
    }                                                                                                          \
  }                                                                                                            \
  extern "C" int fvo_euler_solve_##SUF(void* h, R* U, double gamma, double cfl, double t_end, int max_steps,   \
                                       double* t_out, double* totals) {                                        \
    return euler_solve(*M<R>(h), U, R(gamma), cfl, t_end, max_steps, t_out, totals);                           \
  }                                                                                                            \
  extern "C" double fvo_total_##SUF(void* h, const R* f) { return neumaier_total(*M<R>(h), f); }

FVO_EXPORTS(f64, double)
FVO_EXPORTS(f32, float)

extern "C" int fvo_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

extern "C" void fvo_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
