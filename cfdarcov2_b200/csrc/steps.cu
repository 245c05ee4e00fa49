// Entry points of the time steps: argument checks and dispatch between the
// plain (per-operator, general geometry) and fused paths.
#include "cfdb_internal.hpp"

namespace {

int check_step(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, int path, const char* fn) {
  if (int rc = cfdb_check_mesh(ctx, m)) return rc;
  if (!dtype_ok(dtype)) return cfdb_fail(ctx, CFDB_EINVAL, "%s: unknown dtype %d", fn, dtype);
  if (path != CFDB_PATH_PLAIN && path != CFDB_PATH_FUSED) return cfdb_fail(ctx, CFDB_EINVAL, "%s: unknown path %d", fn, path);
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  return CFDB_OK;
}

}  // namespace

extern "C" int cfdb_heat_step(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, int path, const void* T, void* Tn, double k,
                              double dt) {
  if (int rc = check_step(ctx, m, dtype, path, "cfdb_heat_step")) return rc;
  if (!T || !Tn) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_heat_step: NULL field pointer");
  if (T == Tn) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_heat_step: T and T_next must differ (no in-place stencil writes)");
  if (!std::isfinite(k) || !std::isfinite(dt)) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_heat_step: k and dt must be finite");
  if (path == CFDB_PATH_FUSED) return fused_heat_step(ctx, m, dtype, T, Tn, k, dt);
  if (int rc = cfdb_mesh_need_plain(m, dtype)) return rc;
  PlainGeomDev& p = m->plain[dtype == CFDB_F64 ? 1 : 0];
  if (!p.stab_tmp)
    if (int rc = cfdb_dev_alloc(ctx, int64_t(dtype_size(dtype)) * 18 * m->n, &p.stab_tmp)) return rc;
  if (int rc = plain_lapl(ctx, m, dtype, T, p.stab_tmp, 7)) return rc;
  return plain_heat_update(ctx, dtype, p.stab_tmp, T, k, dt, Tn, m->n);
}

extern "C" int cfdb_heat_step_fixed(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* T, void* Tn, double k,
                                    double dt, const void* fixed) {
  if (int rc = check_step(ctx, m, dtype, CFDB_PATH_FUSED, "cfdb_heat_step_fixed")) return rc;
  if (!T || !Tn || !fixed) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_heat_step_fixed: NULL field pointer");
  if (T == Tn || fixed == Tn)
    return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_heat_step_fixed: T_next must differ from T and the fixed values");
  if (!std::isfinite(k) || !std::isfinite(dt))
    return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_heat_step_fixed: k and dt must be finite");
  return fused_heat_step(ctx, m, dtype, T, Tn, k, dt, fixed);
}

extern "C" int cfdb_d2t_step(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, const void* u, const void* u_prev, void* u_next,
                             double k, const int32_t* masks, int32_t n_terms, double dt, int first_step) {
  if (int rc = check_step(ctx, m, dtype, CFDB_PATH_FUSED, "cfdb_d2t_step")) return rc;
  if (dtype != CFDB_F32) return cfdb_fail(ctx, CFDB_EUNSUPPORTED, "cfdb_d2t_step computes in float32 only");
  if (!u || !u_next || (!first_step && !u_prev)) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_d2t_step: NULL field pointer");
  if (u == u_next || (!first_step && u_prev == u_next))
    return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_d2t_step: u_next must differ from u and u_prev (no in-place stencil writes)");
  if (!masks || n_terms < 1 || n_terms > 3) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_d2t_step: need 1 to 3 terms");
  for (int j = 0; j < n_terms; ++j)
    if (masks[j] < 1 || masks[j] > 7)
      return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_d2t_step: term %d has mask %d (1..7)", j, masks[j]);
  if (!std::isfinite(k) || !std::isfinite(dt)) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_d2t_step: k and dt must be finite");
  return fused_d2t_step(ctx, m, u, first_step ? nullptr : u_prev, u_next, k, masks, n_terms, dt, first_step);
}

extern "C" int cfdb_wave_step(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, int path, const void* q, void* qn,
                              const void* c, double cconst, int mode, double dt) {
  if (int rc = check_step(ctx, m, dtype, path, "cfdb_wave_step")) return rc;
  if (!q || !qn) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_wave_step: NULL state pointer");
  if (q == qn) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_wave_step: q and q_next must differ (no in-place stencil writes)");
  if (mode != 0 && mode != 1) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_wave_step: speed_mode must be 0 or 1");
  if (!c && !(cconst > 0)) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_wave_step: c_const must be > 0");
  if (!std::isfinite(dt)) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_wave_step: dt must be finite");
  if (path == CFDB_PATH_PLAIN) return plain_wave_step(ctx, m, dtype, q, qn, c, cconst, mode, dt);
  if (m->uniform) return fused_wave_step(ctx, m, dtype, q, qn, c, cconst, mode, dt);
  return compact_wave_step(ctx, m, dtype, q, qn, c, cconst, mode, dt);
}

extern "C" int cfdb_wave_adjoint_step(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, int path, const void* q,
                                      const void* lam1, void* lam0, const void* c, void* gc, double dt) {
  if (int rc = check_step(ctx, m, dtype, path, "cfdb_wave_adjoint_step")) return rc;
  if (!q || !lam1 || !lam0 || !c || !gc) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_wave_adjoint_step: NULL pointer");
  if (lam1 == lam0) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_wave_adjoint_step: lam_next and lam_n must differ");
  if (path == CFDB_PATH_FUSED && m->uniform && dtype == CFDB_F32)
    return fused_wave_adjoint(ctx, m, dtype, q, lam1, lam0, c, gc, dt);
  return plain_wave_adjoint(ctx, m, dtype, q, lam1, lam0, c, gc, dt);
}

extern "C" int cfdb_heat_run(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, int path, void* Ta, void* Tb, double k, double dt,
                             int32_t steps, int use_graph, int* final_in_b) {
  CfdbRange range_("cfdb_heat_run");
  if (int rc = check_step(ctx, m, dtype, path, "cfdb_heat_run")) return rc;
  if (!Ta || !Tb || Ta == Tb) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_heat_run: need distinct T_a and T_b");
  if (path == CFDB_PATH_FUSED && dtype == CFDB_F32 && std::isfinite(k) && std::isfinite(dt)) {
    int launched = 0;
    const int r = heat_resident_run(ctx, m, Ta, Tb, k, dt, steps, &launched);
    if (r == CFDB_OK) {
      if (final_in_b) *final_in_b = steps & 1;
      return CFDB_OK;
    }
    if (r != CFDB_EUNSUPPORTED) return r;
  }
  int rc = cfdb_run_steps(
      ctx, Ta, Tb, steps, use_graph,
      [&](const void* src, void* dst) { return cfdb_heat_step(ctx, m, dtype, path, src, dst, k, dt); },
      graph_key("heat", m, dtype, path, Ta, Tb, nullptr, {k, dt}));
  if (!rc && final_in_b) *final_in_b = steps & 1;
  return rc;
}

extern "C" int cfdb_wave_run(cfdb_ctx* ctx, cfdb_mesh* m, int dtype, int path, void* qa, void* qb, const void* c,
                             double cconst, int mode, double dt, int32_t steps, int use_graph, int* final_in_b) {
  CfdbRange range_("cfdb_wave_run");
  if (int rc = check_step(ctx, m, dtype, path, "cfdb_wave_run")) return rc;
  if (!qa || !qb || qa == qb) return cfdb_fail(ctx, CFDB_EINVAL, "cfdb_wave_run: need distinct q_a and q_b");
  int rc = cfdb_run_steps(
      ctx, qa, qb, steps, use_graph,
      [&](const void* src, void* dst) { return cfdb_wave_step(ctx, m, dtype, path, src, dst, c, cconst, mode, dt); },
      graph_key("wave", m, dtype, path, qa, qb, c, {cconst, double(mode), dt}));
  if (!rc && final_in_b) *final_in_b = steps & 1;
  return rc;
}
