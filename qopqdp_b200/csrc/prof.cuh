// prof.cuh -- bracket a launch with CUDA events when profiling is active.
#pragma once
#include "qopb.h"
#include <functional>
#include <vector>

namespace qopb {
int prof_start(const char *name, double bytes);   // -1 when inactive
void prof_stop(int idx);
void prof_discard(int idx);
bool prof_active();

// autotuner: after one warm-up launch of each candidate, times `reps`
// launches of it with CUDA events on the library stream and returns the
// candidate with the least time.  launch(v) must be idempotent (its outputs
// are recomputed by the caller's next real launch).
int tune_pick(const std::vector<int> &cand, const std::function<void(int)> &launch, int reps = 3);

struct ProfScope {
  int idx;
  ProfScope(const char *name, double bytes) : idx(prof_start(name, bytes)) {}
  ~ProfScope() { prof_stop(idx); }
};
}  // namespace qopb
