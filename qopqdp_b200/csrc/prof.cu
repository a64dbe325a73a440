// prof.cu -- per-kernel-class device timing with CUDA events on the library
// stream (QOPB_prof_begin / QOPB_prof_end), plus QOPB_stream.
#include "qopb.h"
#include "prof.cuh"
#include <vector>
#include <string>

namespace qopb {

namespace {
struct Cls { std::string name; double bytes = 0; int launches = 0; double ms = 0; long seen = 0; };
struct Rec { int cls; cudaEvent_t a, b; double bytes; };
struct Prof {
  bool active = false;
  std::vector<Cls> cls;
  std::vector<cudaEvent_t> pool;   // free events
  std::vector<Rec> recs;
  size_t cap = 1 << 16;            // at most this many recorded launches
  int every = 1;                   // bracket every `every`-th launch of a class
};
Prof g_prof;

cudaEvent_t take_event() {
  if (g_prof.pool.empty()) {
    for (int i = 0; i < 256; i++) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); break; }
      g_prof.pool.push_back(e);
    }
    if (g_prof.pool.empty()) return nullptr;
  }
  cudaEvent_t e = g_prof.pool.back();
  g_prof.pool.pop_back();
  return e;
}
}  // namespace

int prof_start(const char *name, double bytes) {
  if (!g_prof.active || g_prof.recs.size() >= g_prof.cap) return -1;
  int c = -1;
  for (size_t i = 0; i < g_prof.cls.size(); i++)
    if (g_prof.cls[i].name == name) { c = (int)i; break; }
  if (c < 0) {
    g_prof.cls.push_back(Cls{name});
    c = (int)g_prof.cls.size() - 1;
  }
  if (g_prof.cls[c].seen++ % g_prof.every != 0) return -1;
  cudaEvent_t a = take_event(), b = take_event();
  if (!a || !b) return -1;
  cudaEventRecord(a, ctx().s);
  g_prof.recs.push_back(Rec{c, a, b, bytes});
  return (int)g_prof.recs.size() - 1;
}

void prof_stop(int idx) {
  if (idx < 0) return;
  cudaEventRecord(g_prof.recs[idx].b, ctx().s);
}

// the launch behind record idx did no work (e.g. it found a stop flag set):
// keep it out of the per-class averages
void prof_discard(int idx) {
  if (idx < 0 || idx >= (int)g_prof.recs.size()) return;
  g_prof.recs[idx].cls = -1;
}

bool prof_active() { return g_prof.active; }

int tune_pick(const std::vector<int> &cand, const std::function<void(int)> &launch, int reps) {
  Context &c = ctx();
  cudaEvent_t a = nullptr, b = nullptr;
  int best = cand.empty() ? -1 : cand[0];
  float best_ms = 3.0e38f;
  try {
    QCHECK(cudaEventCreate(&a));
    QCHECK(cudaEventCreate(&b));
    for (int v : cand) {
      launch(v);   // warm-up
      QCHECK(cudaEventRecord(a, c.s));
      for (int r = 0; r < reps; r++) launch(v);
      QCHECK(cudaEventRecord(b, c.s));
      QCHECK(cudaEventSynchronize(b));
      float ms = 0;
      QCHECK(cudaEventElapsedTime(&ms, a, b));
      if (ms < best_ms) { best_ms = ms; best = v; }
    }
  } catch (...) {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    throw;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return best;
}

}  // namespace qopb

using namespace qopb;

extern "C" void *QOPB_stream(void) {
  try {
    ensure_ready();
  } catch (Fail &) {
    return nullptr;
  }
  return (void *)ctx().s;
}

extern "C" int QOPB_prof_begin(void) {
  g_prof.recs.clear();
  g_prof.cls.clear();
  g_prof.active = true;
  return 0;
}

extern "C" int QOPB_prof_every(int n) {
  if (n < 1) return -1;
  g_prof.every = n;
  return 0;
}

extern "C" int QOPB_prof_end(QOPB_kstat_t *out, int max) {
  g_prof.active = false;
  if (ctx().s) cudaStreamSynchronize(ctx().s);
  for (auto &r : g_prof.recs) {
    float ms = 0;
    if (r.cls < 0) {
      g_prof.pool.push_back(r.a);
      g_prof.pool.push_back(r.b);
      continue;
    }
    if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      g_prof.cls[r.cls].ms += ms;
      g_prof.cls[r.cls].launches += 1;
      g_prof.cls[r.cls].bytes += r.bytes;
    } else {
      cudaGetLastError();
    }
    g_prof.pool.push_back(r.a);
    g_prof.pool.push_back(r.b);
  }
  g_prof.recs.clear();
  int n = (int)g_prof.cls.size();
  for (int i = 0; i < n && i < max && out; i++) {
    memset(out[i].name, 0, sizeof(out[i].name));
    strncpy(out[i].name, g_prof.cls[i].name.c_str(), sizeof(out[i].name) - 1);
    out[i].launches = g_prof.cls[i].launches;
    out[i].total_ms = g_prof.cls[i].ms;
    out[i].bytes_per_launch = g_prof.cls[i].launches ? g_prof.cls[i].bytes / g_prof.cls[i].launches : 0.0;
  }
  return n;
}
