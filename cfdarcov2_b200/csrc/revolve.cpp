// Binomial checkpointing schedule ("revolve", A. Griewank and A. Walther,
// ACM TOMS 26(1), 2000, Alg. 799), written as a recursive split.
//
// With s snapshot slots (one of them holding the segment's first state) and
// r allowed re-advances per step, beta(s, r) = C(s + r, s) steps can be
// reversed.  A segment of l steps takes the smallest r with beta(s, r) >= l,
// advances l1 = min(beta(s, r-1), l - beta(s-1, r-1)) steps, stores a
// snapshot there, reverses the right part with s-1 slots, frees the slot and
// reverses the left part with s slots.  With a single slot every step is recomputed from the segment
// start.  The forward-step count of this schedule equals the optimum
// r l - beta(s+1, r-1) (checked by the tests).
#include <algorithm>
#include <cstdint>
#include <vector>

#include "cfdb_internal.hpp"

namespace {

struct Action { int32_t act, arg, step; };

double beta(int s, int r) {  // C(s + r, s) in double (saturates harmlessly for large arguments)
  double b = 1.0;
  for (int k = 1; k <= s; ++k) b = b * double(r + k) / double(k);
  return b;
}

struct Planner {
  std::vector<Action> out;
  int64_t forward = 0;
  int current = -1;  // step index of the state currently held (-1: unknown)
  std::vector<int> slot_step;  // step stored in each slot (-1 free)

  int slot_of(int step) const {
    for (size_t k = 0; k < slot_step.size(); ++k)
      if (slot_step[k] == step) return int(k);
    return -1;
  }
  int take(int step) {
    for (size_t k = 0; k < slot_step.size(); ++k)
      if (slot_step[k] < 0) {
        slot_step[k] = step;
        out.push_back({CFDB_RV_TAKESHOT, int32_t(k), int32_t(step)});
        return int(k);
      }
    return -1;
  }
  void release(int step) {
    const int k = slot_of(step);
    if (k >= 0) slot_step[k] = -1;
  }
  void go_to(int start) {
    if (current != start) {
      out.push_back({CFDB_RV_RESTORE, int32_t(slot_of(start)), int32_t(start)});
      current = start;
    }
  }
  void advance(int k) {
    if (k <= 0) return;
    out.push_back({CFDB_RV_ADVANCE, int32_t(k), int32_t(current)});
    current += k;
    forward += k;
  }
  void turn(int step, bool first) {
    out.push_back({first ? CFDB_RV_FIRSTURN : CFDB_RV_YOUTURN, 0, int32_t(step)});
    current = -1;  // the adjoint step consumes the state's role
  }

  // Reverse steps [start, end); the state `start` is in a slot; s slots in
  // total are available to this segment (including start's).
  void rev(int start, int end, int s, bool& first) {
    const int l = end - start;
    if (l <= 0) return;
    if (l == 1) {
      go_to(start);
      turn(start, first);
      first = false;
      return;
    }
    if (s <= 1) {
      for (int t = end - 1; t >= start; --t) {
        go_to(start);
        advance(t - start);
        turn(t, first);
        first = false;
      }
      return;
    }
    int r = 0;
    while (beta(s, r) < double(l)) ++r;
    // Optimal split: the left part may be re-advanced r-1 more times
    // (l1 <= beta(s, r-1)) and the right part must still need r repetitions
    // with one slot fewer (l - l1 >= beta(s-1, r-1)).
    const double cap = std::min(beta(s, r - 1), double(l) - beta(s - 1, r - 1));
    const int l1 = int(std::max(1.0, std::min(cap, double(l - 1))));
    const int m = start + l1;
    go_to(start);
    advance(l1);
    take(m);
    rev(m, end, s - 1, first);
    release(m);
    rev(start, m, s, first);
  }
};

}  // namespace

// Shared with the gradient driver.
int cfdb_revolve_build(int32_t steps, int32_t snapshots, std::vector<int32_t>& act, std::vector<int32_t>& arg,
                       std::vector<int32_t>& at, int64_t* forward) {
  Planner p;
  p.slot_step.assign(size_t(snapshots), -1);
  p.slot_step[0] = 0;  // the initial state
  p.out.push_back({CFDB_RV_TAKESHOT, 0, 0});
  p.current = 0;
  bool first = true;
  p.rev(0, steps, snapshots, first);
  act.clear(); arg.clear(); at.clear();
  for (const Action& a : p.out) {
    act.push_back(a.act);
    arg.push_back(a.arg);
    at.push_back(a.step);
  }
  if (forward) *forward = p.forward;
  return CFDB_OK;
}

extern "C" int cfdb_revolve_plan(int32_t steps, int32_t snapshots, int32_t* actions, int32_t* args, int32_t* at_step,
                                 int64_t capacity, int64_t* count, int64_t* forward_steps) {
  if (steps < 1 || snapshots < 1 || capacity < 0 || !count)
    return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_revolve_plan: need steps >= 1, snapshots >= 1 and a count pointer");
  if (snapshots > steps) snapshots = steps;
  std::vector<int32_t> a, g, s;
  int64_t fwd = 0;
  cfdb_revolve_build(steps, snapshots, a, g, s, &fwd);
  *count = int64_t(a.size());
  if (forward_steps) *forward_steps = fwd;
  if (capacity > 0) {
    if (!actions || !args || !at_step) return cfdb_fail(nullptr, CFDB_EINVAL, "cfdb_revolve_plan: NULL output arrays");
    const int64_t n = std::min<int64_t>(capacity, int64_t(a.size()));
    for (int64_t k = 0; k < n; ++k) {
      actions[k] = a[size_t(k)];
      args[k] = g[size_t(k)];
      at_step[k] = s[size_t(k)];
    }
  }
  return CFDB_OK;
}
