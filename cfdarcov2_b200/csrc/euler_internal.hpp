// Shared state of the compressible Euler solver (euler.cu, euler_plain.cu).
//
// The time step lives on the device.  Launch s (counted from cfdb_euler_begin)
// reads the clock slot s%2 and the per-direction maximum signal speeds of ring
// slot s%3 (the state it advances), computes
//   dt = cfl / (lam_x/dx + lam_y/dy + lam_z/dz), clipped onto t_end,
// writes the speeds of the new state into ring slot (s+1)%3 and zeroes slot
// (s+2)%3 for launch s+1, and advances the clock into slot (s+1)%2.  The
// FP64 Neumaier totals of the new state: the plain path's reduction launch
// folds them itself (its last CTA); a fused launch leaves per-CTA partials
// (buffer s%2) and records its step in pending[s%2], and the next launch, or
// cfdb_euler_fold before the host reads the totals, folds them, so no launch
// ends waiting for a fold.  Once t_end is reached every further launch only
// copies the clock forward, so the host can enqueue steps without reading dt
// back (the reference syncs and copies a scalar every step,
// src/fvm3d.cpp:641-662, src/cuda_operators.cu:184-189).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "cfdb_internal.hpp"

struct EulerClock {
  double t[2];
  unsigned long long lam[3][3];  // non-negative doubles as ordered bit patterns
  long long steps[2];
  int finished[2];
  unsigned int counter;  // last-CTA counter of the plain path's reduction, reset by the last CTA
  int pad;
  long long pending[2];  // fused launch s: the step whose partials (buffer s%2) are not folded yet, 0 for none
};

// Neumaier pair, two fields (rho, E).
struct Comp2 {
  double s0, c0, s1, c1;
};

struct cfdb_euler {
  cfdb_ctx* ctx = nullptr;
  cfdb_mesh* mesh = nullptr;
  int dtype = CFDB_F32;
  int path = CFDB_PATH_FUSED;
  double gamma = 1.4, cfl = 0.4, t_end = 0.2;
  int64_t max_steps = 0;
  EulerClock* clock = nullptr;
  double* totals = nullptr;  // 2 * (max_steps + 1)
  Comp2* part = nullptr;     // per-CTA partials: two buffers of part_cap (the fused path alternates them)
  int part_cap = 0;
  int fused_grid = 0;     // CTAs of the last fused launch (the partials it left)
  int fused_threads = 0;  // and their size (the fold runs in the same order)
  int64_t launches = 0;
};

// The host-visible snapshot of the clock after `launches` launches.
inline int euler_slot(int64_t launches) { return int(launches & 1); }

__host__ __device__ inline double euler_dt(const double lam[3], double dx, double dy, double dz, double cfl,
                                           double t, double t_end, bool* last) {
  const double rate = (lam[0] / dx + lam[1] / dy) + lam[2] / dz;
  double dt = cfl / rate;
  *last = false;
  if (dt >= t_end - t) {
    dt = t_end - t;
    *last = true;
  }
  return dt;
}

// euler_plain.cu
int euler_plain_step(cfdb_euler* e, const void* U, void* Un, int64_t s);
int euler_reduce(cfdb_euler* e, const void* U, int64_t s, int begin_mode);
int euler_reduce_grid(const cfdb_euler* e);
// euler.cu
int euler_fused_step(cfdb_euler* e, const void* U, void* Un, int64_t s);
int euler_fused_grid(const cfdb_euler* e);
