// serve.cu -- solve service (B200 addition, no counterpart in the
// reference): callers queue requests, one worker thread groups the systems
// of requests on the same link handle and parity into batched
// mixed-precision solves (batch.cu, up to BATCH_MAX systems) and writes the
// results back in the QOP raw layout with the QOP_asqtad_invert
// normalisation (m A^-1 b).
//
// Requests of one group are taken in arrival order from the front of the
// queue; a request is never split across batches.  Timing per request:
// queue (submit -> batch start), solve (batch start -> results copied) and
// total.  While the service runs the worker owns the library (its global
// stream, current lattice and option state); callers only submit and wait.
#include "solvers.cuh"
#include "fields.cuh"
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
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
  int status = QOP_SUCCESS, iters_max = 0, batch = 0;
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

// one batched solve for a group of requests sharing links, lattice, parity
void run_group(std::vector<Job *> &grp) {
  const QOPB_request_t &r0 = grp[0]->rq;
  if (QOPB_lattice_use(r0.lattice) != 0) fail(QOP_FAIL, "serve: unknown lattice %d", r0.lattice);
  handle_check(r0.links, "FermionLinksAsqtad");
  FlaT<double> *f = reinterpret_cast<FlaT<double> *>(r0.links);
  const int eo = r0.evenodd;
  const Geom &g = ctx().g;
  std::vector<double> m, rq;
  std::vector<c2<double> *> x, b;
  std::vector<std::pair<Job *, int>> who;
  int max_iter = 1;
  for (Job *j : grp) {
    max_iter = std::max(max_iter, j->rq.max_iter > 0 ? j->rq.max_iter : 100000);
    for (int k = 0; k < j->rq.nrhs; k++) {
      m.push_back(j->rq.mass);
      rq.push_back(j->rq.rsqmin);
      who.push_back({j, k});
    }
  }
  const int n = (int)m.size();
  try {
    for (int s = 0; s < n; s++) {
      c2<double> *xs = dalloc<c2<double>>(vec_elems(g)), *bs = dalloc<c2<double>>(vec_elems(g));
      x.push_back(xs);
      b.push_back(bs);
      dzero(xs, sizeof(c2<double>) * vec_elems(g));
      dzero(bs, sizeof(c2<double>) * vec_elems(g));
      raw_to_dev<double, double>(bs, who[s].first->src[who[s].second], 3, eo);
    }
    std::vector<int> its(n);
    std::vector<double> frs(n);
    run_batch(f, eo, n, m.data(), x.data(), b.data(), rq.data(), max_iter, its.data(), frs.data());
    for (int s = 0; s < n; s++) {
      Job *j = who[s].first;
      dev_to_raw<double, double>(j->dst[who[s].second], x[s], 3, eo, m[s]);   // m A^-1 b
      j->iters_max = std::max(j->iters_max, its[s]);
      j->rsq_max = std::max(j->rsq_max, frs[s]);
      j->batch = n;
    }
  } catch (...) {
    for (auto *p : x) dfree(p);
    for (auto *p : b) dfree(p);
    throw;
  }
  for (auto *p : x) dfree(p);
  for (auto *p : b) dfree(p);
  sync();
}

void worker_loop(int device) {
  cudaSetDevice(device);
  Service &S = g_srv;
  while (true) {
    std::vector<Job *> grp;
    {
      std::unique_lock<std::mutex> lk(S.mu);
      S.cv.wait(lk, [&] { return S.stopping || !S.queue.empty(); });
      if (S.queue.empty()) return;   // stopping and drained
      const Job *first = S.queue.front();
      int nsys = 0;
      for (auto it = S.queue.begin(); it != S.queue.end();) {
        const QOPB_request_t &r = (*it)->rq;
        if (r.links == first->rq.links && r.lattice == first->rq.lattice && r.evenodd == first->rq.evenodd &&
            nsys + r.nrhs <= BATCH_MAX) {
          nsys += r.nrhs;
          grp.push_back(*it);
          it = S.queue.erase(it);
        } else {
          ++it;
        }
      }
    }
    const double t0 = now_ms();
    for (Job *j : grp) j->t_start = t0;
    int status = QOP_SUCCESS;
    try {
      run_group(grp);
    } catch (Fail &e) {
      fprintf(stderr, "QOPB serve: %s\n", e.msg.c_str());
      status = e.status;
    }
    {
      std::lock_guard<std::mutex> lk(S.mu);
      const double t1 = now_ms();
      for (Job *j : grp) {
        j->t_done = t1;
        j->status = status;
        j->done = true;
      }
    }
    S.cv_done.notify_all();
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
