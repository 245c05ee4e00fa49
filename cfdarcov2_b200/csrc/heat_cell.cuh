// The fused heat update of one cell, shared by the TMA sweep (one launch per
// step) and the cluster-resident solver (all steps in one launch):
//   T' = T + (cx lx + (cy ly + cz lz)),  l_d = (T_d+ - T) + (T_d- - T)
// with c_d = dt k / h_d^2 and a wall neighbour equal to the cell itself
// (zero gradient: the reference's boundary faces point to the cell,
// src/mesh3d.cpp:273-276).  Every operation is an explicitly rounded
// intrinsic (two fused multiply-adds, the rest separate), so the compiler's
// contraction choices, which differ between the two kernels, cannot change
// the result: both paths give the same bits.
#pragma once

__device__ __forceinline__ float heat_update(float t, float xm, float xp, float ym, float yp, float zm, float zp,
                                             float cx, float cy, float cz) {
  const float lx = __fadd_rn(__fsub_rn(xp, t), __fsub_rn(xm, t));
  const float ly = __fadd_rn(__fsub_rn(yp, t), __fsub_rn(ym, t));
  const float lz = __fadd_rn(__fsub_rn(zp, t), __fsub_rn(zm, t));
  return __fadd_rn(t, __fmaf_rn(cx, lx, __fmaf_rn(cy, ly, __fmul_rn(cz, lz))));
}
