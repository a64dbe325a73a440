// prof.cuh -- bracket a launch with CUDA events when profiling is active.
#pragma once
#include "qopb.h"

namespace qopb {
int prof_start(const char *name, double bytes);   // -1 when inactive
void prof_stop(int idx);
void prof_discard(int idx);
bool prof_active();

struct ProfScope {
  int idx;
  ProfScope(const char *name, double bytes) : idx(prof_start(name, bytes)) {}
  ~ProfScope() { prof_stop(idx); }
};
}  // namespace qopb
