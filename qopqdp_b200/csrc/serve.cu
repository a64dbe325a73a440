// serve.cu -- solve service (B200 addition, no counterpart in the
// reference) with continuous batching: callers queue requests; one worker
// thread keeps a batched mixed-precision solver (BatchEngine, batch.cu: 16
// slots) per link handle and parity in flight and admits the systems of a
// queued request into free slots between solver steps, so a request that
// arrives while others are on the GPU joins their hop launches at once
// instead of waiting for their batch to finish.  A step advances every
// running system of one engine by a chunk of iterations plus its reliable
// updates.  Each engine runs on a stream of its own and the worker launches
// the chunks of all engines with work before it collects any, so requests
// on different lattices or handles run on the device side by side.  Results
// are written
// back in the QOP raw layout with the QOP_asqtad_invert normalisation (m
// A^-1 b) as each system finishes.
//
// Option serve_policy 1 steps only the engine holding the oldest request
// (requests still join any engine's free slots): first-come first-served
// across engines, which shortens the longest latencies of a heavy-tailed
// mix at the cost of the median.
//
// Admission: requests in arrival order; a request is never split (all of
// its sources enter one engine together) and a request that does not fit
// holds back the later requests of its engine.  A new engine is created
// only if its device memory fits in the free HBM (less a reserve) while
// other engines run, and within the option serve_hbm_mb when it is set;
// an engine whose slots are all free is destroyed.  A request whose source
// holds a NaN or Inf fails alone (QOP_FAIL) before it takes a slot.
// Timing per request: queue (submit -> admission), solve (admission ->
// last source finished) and total.  While the service runs the worker owns
// the library (its global stream, current lattice and option state);
// callers only submit and wait.
#include "solvers.cuh"
#include "fields.cuh"
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

namespace qopb {
namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Job {
  long long id = 0;
  QOPB_request_t rq{};
  std::vector<const double *> src;
  std::vector<double *> dst;
  double t_submit = 0, t_start = 0, t_done = 0;
  int status = QOP_SUCCESS, iters_max = 0, batch = 0, left = 0;
  double rsq_max = 0;
  bool done = false;
};

struct Service {
  std::mutex mu;
  std::condition_variable cv, cv_done;
  std::deque<Job *> queue;
  std::unordered_map<long long, Job *> jobs;
  std::thread worker;
  bool running = false, stopping = false;
  long long next = 0;
};
Service g_srv;

// one engine with its FP64 solution and source vectors per slot
struct Lane {
  int lattice = 0, eo = 0;
  size_t bytes = 0;            // device memory of the engine and its vectors
  const void *links = nullptr;
  std::unique_ptr<BatchEngine> eng;
  std::vector<c2<double> *> x, b;
  struct Occ { Job *job = nullptr; int k = 0; };
  std::vector<Occ> occ;
  ~Lane() {
    eng.reset();
    for (auto *p : x) dfree(p);
    for (auto *p : b) dfree(p);
  }
};

constexpr size_t HBM_RESERVE = size_t(2) << 30;   // left free when other engines run

// free device memory, counting what the stream-ordered pool holds unused
size_t free_hbm() {
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) { cudaGetLastError(); return 0; }
  cudaMemPool_t pool;
  uint64_t reserved = 0, used = 0;
  if (cudaDeviceGetDefaultMemPool(&pool, ctx().device) == cudaSuccess &&
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
    fr += (size_t)(reserved - used);
  cudaGetLastError();
  return fr;
}

void finish(Job *j, int status) {
  Service &S = g_srv;
  {
    std::lock_guard<std::mutex> lk(S.mu);
    j->t_done = now_ms();
    if (status != QOP_SUCCESS) j->status = status;
    j->done = true;
  }
  S.cv_done.notify_all();
}

struct Worker {
  std::vector<std::unique_ptr<Lane>> lanes;
  std::deque<Job *> pending;   // taken from the queue, not yet admitted

  Lane *find(const QOPB_request_t &r) {
    for (auto &l : lanes)
      if (l->links == r.links && l->lattice == r.lattice && l->eo == r.evenodd) return l.get();
    return nullptr;
  }
  bool any_running() const {
    for (auto &l : lanes)
      if (l->eng->busy() > 0) return true;
    return false;
  }

  // a new engine for the request's handle and parity on the current lattice;
  // nullptr (nothing allocated) when it does not fit while others run
  Lane *create(const QOPB_request_t &r) {
    const Geom &g = ctx().g;
    const size_t need = BatchEngine::bytes(g, BATCH_MAX) + 2 * sizeof(c2<double>) * vec_elems(g) * BATCH_MAX;
    if (any_running() && free_hbm() < need + HBM_RESERVE) return nullptr;
    // option serve_hbm_mb: the engines together stay within the budget (a
    // lone engine is always admitted, so that every request can run)
    const double budget = ctx().opt.serve_hbm_mb * 1048576.0;
    size_t held = 0;
    for (auto &o : lanes) held += o->bytes;
    if (budget > 0 && !lanes.empty() && (double)(held + need) > budget) return nullptr;
    auto l = std::make_unique<Lane>();
    l->bytes = need;
    l->lattice = r.lattice;
    l->eo = r.evenodd;
    l->links = r.links;
    l->eng = std::make_unique<BatchEngine>(reinterpret_cast<FlaT<double> *>(r.links), r.evenodd, BATCH_MAX, true);
    for (int s = 0; s < BATCH_MAX; s++) {
      l->x.push_back(dalloc<c2<double>>(vec_elems(g)));
      l->b.push_back(dalloc<c2<double>>(vec_elems(g)));
    }
    sync();   // allocated before the engine's stream uses them
    l->occ.assign(BATCH_MAX, Lane::Occ{});
    lanes.push_back(std::move(l));
    return lanes.back().get();
  }

  // admit pending requests in arrival order while slots and memory allow
  void admit() {
    std::vector<const Lane *> held;   // engines whose earlier request did not fit
    std::vector<std::tuple<const void *, int, int>> held_new;
    for (auto it = pending.begin(); it != pending.end();) {
      Job *j = *it;
      const QOPB_request_t &r = j->rq;
      const auto key = std::make_tuple((const void *)r.links, r.lattice, (int)r.evenodd);
      bool later = false;
      for (auto &k : held_new) later = later || k == key;
      Lane *l = find(r);
      if (later || (l && std::find(held.begin(), held.end(), l) != held.end())) { ++it; continue; }
      bool starting = false;   // slots of l are being filled
      try {
        if (QOPB_lattice_use(r.lattice) != 0) fail(QOP_FAIL, "serve: unknown lattice %d", r.lattice);
        handle_check(r.links, "FermionLinksAsqtad");
        if (!l) {
          try {
            l = create(r);
          } catch (Fail &e) {
            if (e.status != QOP_MEM_ERROR || !any_running()) throw;
            l = nullptr;
          }
          if (!l) {   // waits for memory
            held_new.push_back(key);
            ++it;
            continue;
          }
        }
        if (BATCH_MAX - l->eng->busy() < r.nrhs) {
          held.push_back(l);
          ++it;
          continue;
        }
        const Geom &g = ctx().g;
        // a source with NaN or Inf fails its own request, before it holds a slot
        for (int k = 0; k < r.nrhs; k++) {
          const double *src = j->src[k];
          double acc = 0;
          for (i64 e = 0; e < 6 * g.V; e++) acc += src[e] * 0.0;   // NaN or Inf -> NaN
          need_finite(acc, "serve: source");
        }
        j->t_start = now_ms();
        j->left = r.nrhs;
        starting = true;
        StreamScope ss(l->eng->stream());
        for (int k = 0; k < r.nrhs; k++) {
          const int s = l->eng->free_slot();
          dzero(l->b[s], sizeof(c2<double>) * vec_elems(g));
          raw_to_dev<double, double>(l->b[s], j->src[k], 3, r.evenodd);
          l->occ[s] = Lane::Occ{j, k};
          l->eng->start(s, l->x[s], l->b[s], r.mass, r.rsqmin, r.max_iter > 0 ? r.max_iter : 100000, true);
        }
        j->batch = std::max(j->batch, l->eng->busy());
      } catch (Fail &e) {
        fprintf(stderr, "QOPB serve: %s\n", e.msg.c_str());
        bool in_lane = false;
        if (starting) {
          // the engine's state is unknown after a failed start: every request
          // in it fails (this one too, if it holds a slot)
          for (auto &o : l->occ) in_lane = in_lane || o.job == j;
          drop(l, e.status);
        }
        if (!in_lane) {
          j->t_start = now_ms();
          finish(j, e.status);
        }
      }
      it = pending.erase(it);
    }
  }

  // fail every request with a source in lane l and destroy it
  void drop(Lane *l, int status) {
    std::vector<Job *> js;
    for (auto &o : l->occ)
      if (o.job && std::find(js.begin(), js.end(), o.job) == js.end()) js.push_back(o.job);
    for (auto &p : lanes)
      if (p.get() == l) { p.reset(); break; }
    lanes.erase(std::remove(lanes.begin(), lanes.end(), nullptr), lanes.end());
    for (Job *j : js) finish(j, status);
  }

  // submission time of the oldest request holding a slot of l
  static double oldest(const Lane *l) {
    double t = 1e300;
    for (auto &o : l->occ)
      if (o.job) t = std::min(t, o.job->t_submit);
    return t;
  }

  // one step of every engine with work (policy 1: of the engine holding the
  // oldest request, and of engines with nothing left to iterate): every
  // engine's chunk is launched on its own stream before any is collected,
  // so the chunks of different lattices run side by side; then results of
  // finished systems
  void step_all() {
    const Lane *first = nullptr;
    if (ctx().opt.serve_policy == 1)
      for (auto &l : lanes)
        if (l->eng->running() > 0 && (!first || oldest(l.get()) < oldest(first))) first = l.get();
    std::vector<Lane *> go;
    for (auto &l : lanes)
      if (l->eng->busy() > 0 && !(first && l.get() != first && l->eng->running() > 0)) go.push_back(l.get());
    std::vector<Lane *> launched;
    for (Lane *l : go) {
      try {
        if (QOPB_lattice_use(l->lattice) != 0) fail(QOP_FAIL, "serve: unknown lattice %d", l->lattice);
        l->eng->launch();
        launched.push_back(l);
      } catch (Fail &e) {
        fprintf(stderr, "QOPB serve: %s\n", e.msg.c_str());
        drop(l, e.status);
      }
    }
    for (Lane *l : launched) {
      std::vector<Job *> ended;
      try {
        if (QOPB_lattice_use(l->lattice) != 0) fail(QOP_FAIL, "serve: unknown lattice %d", l->lattice);
        const std::vector<int> fin = l->eng->collect();
        const int nb = l->eng->busy();
        for (auto &o : l->occ)
          if (o.job) o.job->batch = std::max(o.job->batch, nb);
        StreamScope ss(l->eng->stream());
        for (int s : fin) {
          Lane::Occ &o = l->occ[s];
          Job *j = o.job;
          const QOPB_request_t &r = j->rq;
          dev_to_raw<double, double>(j->dst[o.k], l->x[s], 3, r.evenodd, r.mass);   // m A^-1 b
          j->iters_max = std::max(j->iters_max, l->eng->iters(s));
          j->rsq_max = std::max(j->rsq_max, l->eng->final_rsq(s));
          l->eng->release(s);
          o = Lane::Occ{};
          if (--j->left == 0) ended.push_back(j);
        }
        if (!ended.empty()) sync();
      } catch (Fail &e) {
        fprintf(stderr, "QOPB serve: %s\n", e.msg.c_str());
        for (Job *j : ended) finish(j, QOP_SUCCESS);
        drop(l, e.status);
        continue;
      }
      for (Job *j : ended) finish(j, QOP_SUCCESS);
    }
    // engines with no system left are freed (their memory goes to new ones)
    lanes.erase(std::remove_if(lanes.begin(), lanes.end(), [](const std::unique_ptr<Lane> &l) {
                  return l->eng->busy() == 0;
                }),
                lanes.end());
  }
};

void worker_loop(int device) {
  cudaSetDevice(device);
  Service &S = g_srv;
  Worker w;
  while (true) {
    {
      std::unique_lock<std::mutex> lk(S.mu);
      const bool work = w.any_running() || !w.pending.empty();
      if (!work) S.cv.wait(lk, [&] { return S.stopping || !S.queue.empty(); });
      while (!S.queue.empty()) {
        w.pending.push_back(S.queue.front());
        S.queue.pop_front();
      }
      if (S.stopping && w.pending.empty() && !w.any_running()) return;
    }
    w.admit();
    if (!w.any_running() && !w.pending.empty()) {
      // nothing runs and the front requests still do not fit: they cannot
      for (Job *j : w.pending) {
        j->t_start = now_ms();
        finish(j, QOP_MEM_ERROR);
      }
      w.pending.clear();
    }
    w.step_all();
  }
}

}  // namespace
}  // namespace qopb

using namespace qopb;

extern "C" {

int QOPB_serve_start(void) {
  Service &S = g_srv;
  std::lock_guard<std::mutex> lk(S.mu);
  if (S.running || !ctx().inited || ctx().dd) return -1;
  try {
    ensure_ready();
  } catch (Fail &) {
    return -1;
  }
  S.stopping = false;
  S.running = true;
  S.worker = std::thread(worker_loop, ctx().device);
  return 0;
}

long long QOPB_serve_submit(const QOPB_request_t *req) {
  Service &S = g_srv;
  if (!req || !req->links || !req->src || !req->dst || req->nrhs < 1 || req->nrhs > BATCH_MAX) return -1;
  if (req->evenodd != QOP_EVEN && req->evenodd != QOP_ODD) return -1;
  if (req->lattice < 0 || req->lattice >= (int)ctx().lats.size() || !(req->rsqmin >= 0)) return -1;
  Job *j = new Job();
  j->rq = *req;
  for (int k = 0; k < req->nrhs; k++) {
    if (!req->src[k] || !req->dst[k]) { delete j; return -1; }
    j->src.push_back(req->src[k]);
    j->dst.push_back(req->dst[k]);
  }
  std::lock_guard<std::mutex> lk(S.mu);
  if (!S.running || S.stopping) { delete j; return -1; }
  j->id = S.next++;
  j->t_submit = now_ms();
  S.jobs[j->id] = j;
  S.queue.push_back(j);
  S.cv.notify_one();
  return j->id;
}

int QOPB_serve_wait(long long ticket, double timeout_s, QOPB_result_t *res) {
  Service &S = g_srv;
  std::unique_lock<std::mutex> lk(S.mu);
  auto it = S.jobs.find(ticket);
  if (it == S.jobs.end()) return -1;
  Job *j = it->second;
  const auto limit = std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 1e9);
  if (!S.cv_done.wait_for(lk, limit, [&] { return j->done; })) return 1;
  if (res) {
    res->status = j->status;
    res->iters_max = j->iters_max;
    res->final_rsq_max = j->rsq_max;
    res->queue_ms = j->t_start - j->t_submit;
    res->solve_ms = j->t_done - j->t_start;
    res->total_ms = j->t_done - j->t_submit;
    res->batch_systems = j->batch;
  }
  S.jobs.erase(it);
  delete j;
  return 0;
}

int QOPB_serve_stop(void) {
  Service &S = g_srv;
  {
    std::lock_guard<std::mutex> lk(S.mu);
    if (!S.running) return -1;
    S.stopping = true;
  }
  S.cv.notify_all();
  S.worker.join();
  std::lock_guard<std::mutex> lk(S.mu);
  S.running = false;
  return 0;
}

}  // extern "C"
