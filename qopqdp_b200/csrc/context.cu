// context.cu -- library state, QOP_init/finalize, options, allocation.
// Reference: lib/common.c:39-191 (init, version, verbosity, raw index),
// lib/asqtad_invert.c:9-113 (inverter options), lib/hisq_links.c:32-78.
#include "qopb.h"
#include <atomic>
#include <cstdarg>
#include <sys/time.h>
#include <mutex>
#include <unordered_map>

namespace qopb {

static Context g_ctx;
Context &ctx() { return g_ctx; }

void check_cuda(cudaError_t e, const char *what, const char *file, int line) {
  if (e == cudaSuccess) return;
  cudaGetLastError();   // clear sticky-free errors
  char buf[512];
  snprintf(buf, sizeof buf, "CUDA error '%s' in %s (%s:%d)", cudaGetErrorString(e), what, file, line);
  throw Fail(e == cudaErrorMemoryAllocation ? QOP_MEM_ERROR : QOP_FAIL, buf);
}

static unsigned long long g_launches = 0;
void count_launches(int n) { g_launches += (unsigned long long)n; }
unsigned long long launch_count() { return g_launches; }

void fail(QOP_status_t s, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  throw Fail(s, buf);
}

void log0(int level, const char *fmt, ...) {
  if (g_ctx.verbosity < level) return;
  va_list ap;
  va_start(ap, fmt);
  vprintf(fmt, ap);
  va_end(ap);
  fflush(stdout);
}

double wtime() {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

void require_init(const char *fn) {
  if (!g_ctx.inited) fail(QOP_FAIL, "%s: QOP_init has not been called", fn);
}

void ensure_ready() {
  Context &c = g_ctx;
  if (c.s) return;
  QCHECK(cudaGetDevice(&c.device));
  QCHECK(cudaStreamCreateWithFlags(&c.s, cudaStreamNonBlocking));
  int sms = 0;
  QCHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device));
  c.red_blocks = sms * 8;
  c.part_cap = (size_t)8 * c.red_blocks;
  QCHECK(cudaMalloc(&c.d_part, sizeof(double) * c.part_cap));
  QCHECK(cudaMalloc(&c.d_count, sizeof(unsigned) * 4));
  QCHECK(cudaMemset(c.d_count, 0, sizeof(unsigned) * 4));
  QCHECK(cudaMalloc(&c.d_res, sizeof(double) * 64));
  QCHECK(cudaMallocHost(&c.h_res, sizeof(double) * 64));
  // keep freed blocks cached in the stream-ordered pool
  cudaMemPool_t pool;
  QCHECK(cudaDeviceGetDefaultMemPool(&pool, c.device));
  uint64_t thr = UINT64_MAX;
  QCHECK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
}

// allocation-failure injection (QOPB_inject_alloc_failure): the n-th
// allocation from now on fails as an out-of-memory would
static std::atomic<int> g_alloc_fail_in{0};

void *dmalloc(size_t bytes) {
  ensure_ready();
  void *p = nullptr;
  if (bytes == 0) bytes = 16;
  if (g_alloc_fail_in.load() > 0 && g_alloc_fail_in.fetch_sub(1) == 1)
    fail(QOP_MEM_ERROR, "device allocation of %zu bytes failed: injected failure", bytes);
  cudaError_t e = cudaMallocAsync(&p, bytes, g_ctx.s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    fail(QOP_MEM_ERROR, "device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
  }
  return p;
}
void dfree(void *p) {
  if (p && g_ctx.s) cudaFreeAsync(p, g_ctx.s);
}
void dzero(void *p, size_t bytes) { QCHECK(cudaMemsetAsync(p, 0, bytes, g_ctx.s)); }
void sync() { QCHECK(cudaStreamSynchronize(g_ctx.s)); }

static std::mutex g_hmu;
static std::unordered_map<const void *, int> g_handles;
void handle_register(const void *h) {
  std::lock_guard<std::mutex> lk(g_hmu);
  g_handles[h] = g_ctx.lat;
}
void handle_forget(const void *h) {
  std::lock_guard<std::mutex> lk(g_hmu);
  g_handles.erase(h);
}
void handle_check(const void *h, const char *what) {
  if (!h) fail(QOP_FAIL, "NULL %s handle", what);
  int lat = -1;
  {
    std::lock_guard<std::mutex> lk(g_hmu);
    auto it = g_handles.find(h);
    if (it != g_handles.end()) lat = it->second;
  }
  if (lat < 0) fail(QOP_FAIL, "%s handle is not a live handle of this library", what);
  if (lat != g_ctx.lat)
    fail(QOP_FAIL, "%s handle belongs to lattice %d, the current lattice is %d", what, lat, g_ctx.lat);
}

// extents even and >= 4 (eo preconditioning and the 3-hop Naik term), V < 2^31
static bool make_geom(const int *ls, Geom &g, bool global = false) {
  g = Geom{};
  g.V = 1;
  for (int i = 0; i < 4; i++) {
    if (ls[i] < 4 || (ls[i] & 1)) {
      fprintf(stderr, "QOP: extent %d in direction %d must be even and >= 4\n", ls[i], i);
      return false;
    }
    g.L[i] = ls[i];
    g.GL[i] = ls[i];
    g.O[i] = 0;
    g.V *= ls[i];
  }
  g.Vh = g.V / 2;
  if (!global && g.V >= (1LL << 31)) {
    fprintf(stderr, "QOP: volume too large for one device\n");
    return false;
  }
  return true;
}

// fused reductions run one block per 64+ sites with up to 4 sums each
static void ensure_partials(const Geom &g) {
  Context &c = g_ctx;
  size_t need = (size_t)4 * (g.Vh / 64 + 64);
  if (need > c.part_cap) {
    QCHECK(cudaStreamSynchronize(c.s));
    QCHECK(cudaFree(c.d_part));
    QCHECK(cudaMalloc(&c.d_part, sizeof(double) * need));
    c.part_cap = need;
  }
}

int grid_for(i64 n, int block) {
  i64 b = (n + block - 1) / block;
  if (b < 1) b = 1;
  if (b > 0x7fffffff) b = 0x7fffffff;
  return (int)b;
}

}  // namespace qopb

using namespace qopb;

#define OPT_TRY try {
#define OPT_CATCH(ret) } catch (Fail &e) { log0(0, "QOP error: %s\n", e.msg.c_str()); return ret; }

extern "C" {

QOP_status_t QOP_init(QOP_layout_t *layout) {
  Context &c = ctx();
  if (c.inited) return QOP_FAIL;
  if (!layout || layout->latdim != 4 || !layout->latsize) {
    fprintf(stderr, "QOP_init: only 4-dimensional lattices are supported\n");
    return QOP_FAIL;
  }
  Geom g{};
  if (!make_geom(layout->latsize, g, true)) return QOP_FAIL;
  OPT_TRY
  ensure_ready();
  // a machine size (or a communicator of several processes) decomposes the
  // lattice; g becomes this process's block
  if (!dd_setup(layout, g)) return QOP_FAIL;
  if (g.V >= (1LL << 31)) {
    fprintf(stderr, "QOP: volume too large for one device\n");
    dd_free();
    return QOP_FAIL;
  }
  ensure_partials(g);
  } catch (Fail &e) {
    log0(0, "QOP error: %s\n", e.msg.c_str());
    dd_free();   // a decomposition set up before the failure
    return QOP_FAIL;
  }
  c.g = g;
  c.lats.assign(1, g);
  c.lat = 0;
  c.verbosity = 0;
  c.proflevel = 0;
  c.inited = 1;
  return QOP_SUCCESS;
}

int QOPB_lattice_create(const int latsize[4]) {
  Context &c = ctx();
  if (!c.inited || !latsize || c.dd) return -1;
  Geom g{};
  if (!make_geom(latsize, g)) return -1;
  OPT_TRY
  ensure_partials(g);
  OPT_CATCH(-1)
  c.lats.push_back(g);
  return (int)c.lats.size() - 1;
}

int QOPB_lattice_use(int id) {
  Context &c = ctx();
  if (!c.inited || id < 0 || id >= (int)c.lats.size()) return -1;
  c.lat = id;
  c.g = c.lats[id];
  return 0;
}

int QOPB_lattice_current(void) { return ctx().inited ? ctx().lat : -1; }

QOP_status_t QOP_finalize(void) {
  Context &c = ctx();
  if (!c.inited) return QOP_FAIL;
  if (c.s) cudaStreamSynchronize(c.s);
  dd_free();
  c.inited = 0;
  return QOP_SUCCESS;
}

int QOP_is_initialized(void) { return ctx().inited; }

unsigned long long QOPB_launch_count(void) { return launch_count(); }

int QOPB_inject_alloc_failure(int n) {
  if (n < 0) return -1;
  g_alloc_fail_in.store(n);
  return 0;
}

const char *QOP_version_str(void) { return "0.21.1-b200"; }
int QOP_version_int(void) { return (0 * 1000 + 21) * 1000 + 1; }

int QOP_verbose(int level) {
  int old = ctx().verbosity;
  ctx().verbosity = level;
  return old;
}
int QOP_profcontrol(int level) {
  int old = ctx().proflevel;
  ctx().proflevel = level;
  return old;
}

// the process holding a site (lib/common.c:134-139); 0 unless decomposed
int QOP_node_number_raw(int coords[]) { return ctx().inited ? dd_node_number(coords) : -1; }

// raw index of a site: even sites first (lib/layout_user.c:237-258)
static int raw_index(const int x[]) {
  const Geom &g = ctx().g;
  i64 l = 0;
  int s = 0;
  for (int i = 0; i < 4; i++) { l = l * g.L[i] + x[i]; s += x[i]; }
  return (int)((s & 1) ? (l + g.V) / 2 : l / 2);
}
// node-local raw index of a site given by global coordinates
static int node_index(const int x[]) { return ctx().dd ? (int)dd_node_index(x) : raw_index(x); }
int QOP_node_index_raw_V(int coords[], QOP_evenodd_t eo) { (void)eo; return ctx().inited ? node_index(coords) : -1; }
int QOP_node_index_raw_G(int coords[], QOP_evenodd_t eo) { (void)eo; return ctx().inited ? node_index(coords) : -1; }
int QOP_sites_on_node_raw_V(QOP_evenodd_t eo) { (void)eo; return (int)ctx().g.V; }
int QOP_sites_on_node_raw_G(QOP_evenodd_t eo) { (void)eo; return (int)ctx().g.V; }

// tags: st, ns, nm, cg, eigcg_nev, eigcg_m, eigcg_l (reference) and
// prec_sloppy (64|32|16), half_format, hop_kernel, recon_long, multi_shift,
// batch_tail, ms_stop, ru_delta, chunk (B200 additions)
QOP_status_t QOP_asqtad_invert_set_opts(QOP_opt_t opts[], int nopts) {
  Options &o = ctx().opt;
  int st = o.style, ns = o.nsvec, nm = o.nvec;
  auto valid_nv = [](int nv, int s) { return nv == 1 || nv == 2 || nv == 4 || nv == 8 || (s == 1 && nv == 16); };
  for (int i = 0; i < nopts; i++)
    if (opts[i].tag && !strcmp(opts[i].tag, "st")) st = (int)opts[i].value;
  if (st < 0 || st > 3) return QOP_FAIL;
  if (!valid_nv(ns, st)) ns = ns < 1 ? 1 : 8;
  if (!valid_nv(nm, st)) nm = nm < 1 ? 1 : 8;
  Options n = o;
  for (int i = 0; i < nopts; i++) {
    const char *t = opts[i].tag;
    double v = opts[i].value;
    if (!t) continue;
    if (!strcmp(t, "ns")) ns = (int)v;
    else if (!strcmp(t, "nm")) nm = (int)v;
    else if (!strcmp(t, "cg")) n.cgtype = (int)v;
    else if (!strcmp(t, "eigcg_nev")) n.eigcg_nev = (int)v;
    else if (!strcmp(t, "eigcg_m")) n.eigcg_m = (int)v;
    else if (!strcmp(t, "eigcg_l")) n.eigcg_numax = (int)v;
    else if (!strcmp(t, "prec_sloppy")) {
      int p = (int)v;
      if (p != 16 && p != 32 && p != 64) return QOP_FAIL;
      n.sloppy_prec = p;
    } else if (!strcmp(t, "batch_kernel")) {
      if (v < -2 || v > 16) return QOP_FAIL;   // 16: the tensor-core hop (bmma.cu)
      n.batch_kernel = (int)v;
    } else if (!strcmp(t, "multi_shift")) {
      n.multi_shift = v != 0;
    } else if (!strcmp(t, "fuse_update")) {
      n.fuse_update = v != 0;
    } else if (!strcmp(t, "batch_tail")) {
      n.batch_tail = v != 0;
    } else if (!strcmp(t, "ms_stop")) {
      if (!(v == -1 || (v >= 0 && v < 1))) return QOP_FAIL;
      n.ms_stop = v;
    } else if (!strcmp(t, "pdl")) {
      n.pdl = v != 0;
    } else if (!strcmp(t, "serve_policy")) {
      if (v != 0 && v != 1) return QOP_FAIL;
      n.serve_policy = (int)v;
    } else if (!strcmp(t, "serve_hbm_mb")) {
      if (!(v >= 0)) return QOP_FAIL;
      n.serve_hbm_mb = v;
    } else if (!strcmp(t, "mbar_tries")) {
      if (v < 0 || v > (1 << 26)) return QOP_FAIL;
      n.mbar_tries = (int)v;
    } else if (!strcmp(t, "recon_long")) {
      n.recon_long = v != 0;
    } else if (!strcmp(t, "hop_kernel")) {
      if (v < -1 || v > 31) return QOP_FAIL;
      n.hop_kernel = (int)v;
    } else if (!strcmp(t, "half_format")) {
      if (v < 0 || v > 2) return QOP_FAIL;
      n.half_format = (int)v;
    } else if (!strcmp(t, "ru_delta")) {
      if (!(v > 0 && v < 1)) return QOP_FAIL;
      n.ru_delta = v;
    } else if (!strcmp(t, "chunk")) {
      if (v < 1 || v > 1024) return QOP_FAIL;
      n.chunk = (int)v;
    }
  }
  if (!valid_nv(ns, st) || !valid_nv(nm, st)) return QOP_FAIL;
  n.style = st; n.nsvec = ns; n.nvec = nm;
  o = n;
  return QOP_SUCCESS;
}

QOP_status_t QOP_hisq_invert_set_opts(QOP_opt_t opts[], int nopts) {
  return QOP_asqtad_invert_set_opts(opts, nopts);
}

QOP_status_t QOP_hisq_links_set_opts(QOP_opt_t opts[], int nopts) {
  Options &o = ctx().opt;
  for (int i = 0; i < nopts; i++) {
    const char *t = opts[i].tag;
    double v = opts[i].value;
    if (!t) continue;
    if (!strcmp(t, "want_deps")) o.want_deps = (int)v;
    else if (!strcmp(t, "want_aux")) o.want_aux = (int)v;
    else if (!strcmp(t, "reunit_allow_svd")) o.reunit_allow_svd = (int)v;
    else if (!strcmp(t, "reunit_svd_only")) o.reunit_svd_only = (int)v;
    else if (!strcmp(t, "reunit_svd_rel_error")) o.reunit_svd_rel_error = v;
    else if (!strcmp(t, "reunit_svd_abs_error")) o.reunit_svd_abs_error = v;
    else if (!strcmp(t, "svd_values_info")) o.svd_values_info = (int)v;
    else if (!strcmp(t, "use_fat7_lepage")) o.use_fat7_lepage = (int)v;
  }
  return QOP_SUCCESS;
}

}  // extern "C"
