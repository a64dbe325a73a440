// dd.cu -- the lattice decomposed over processes, one GPU each.
// Reference: QDP's hypercubic even/odd layout that QOP installs
// (lib/layout_user.c:79-258: the split of the lattice into blocks, the node
// of a site and its node-local index) and lib/common.c:40-83, :134-166
// (QOP_init with a machine size, QOP_node_number_raw, QOP_node_index_raw).
// The reference moves halos and sums reductions through QDP/QMP; here the
// hop kernels read halos that one NCCL group exchanges per hop (dd.cuh), and
// the reductions end with one NCCL all-reduce of their FP64 sums on the
// device.  NCCL is loaded when a communicator is made, so single-GPU use
// never touches it.
#include "qopb.h"
#include "dslash.cuh"
#include "dd.cuh"
#include "mixed.cuh"
#include <dlfcn.h>
#include <nccl.h>

namespace qopb {

// ---------------------------------------------------------------- NCCL
namespace {

struct NcclApi {
  bool loaded = false;
  ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*AllReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  const char *(*GetErrorString)(ncclResult_t) = nullptr;
};
NcclApi g_nccl;

template <typename F> void sym(void *h, const char *name, F &fp) {
  fp = reinterpret_cast<F>(dlsym(h, name));
  if (!fp) fail(QOP_FAIL, "NCCL symbol %s not found", name);
}

// the process's libnccl.so.2 (the one PyTorch loaded, when it did)
void nccl_load() {
  if (g_nccl.loaded) return;
  void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
  if (!h) fail(QOP_FAIL, "cannot load libnccl.so.2: %s", dlerror());
  sym(h, "ncclGetUniqueId", g_nccl.GetUniqueId);
  sym(h, "ncclCommInitRank", g_nccl.CommInitRank);
  sym(h, "ncclCommDestroy", g_nccl.CommDestroy);
  sym(h, "ncclGroupStart", g_nccl.GroupStart);
  sym(h, "ncclGroupEnd", g_nccl.GroupEnd);
  sym(h, "ncclSend", g_nccl.Send);
  sym(h, "ncclRecv", g_nccl.Recv);
  sym(h, "ncclAllReduce", g_nccl.AllReduce);
  sym(h, "ncclGetErrorString", g_nccl.GetErrorString);
  g_nccl.loaded = true;
}

void ncheck(ncclResult_t r, const char *what) {
  if (r != ncclSuccess) fail(QOP_FAIL, "%s: %s", what, g_nccl.GetErrorString(r));
}

struct Comm {
  ncclComm_t comm = nullptr;
  int nranks = 1, rank = 0;
};
Comm g_comm;
int g_self_split = 0;   // directions decomposed with the process as its own neighbour

}  // namespace

// ---------------------------------------------------------------- layout
// The reference's split of the lattice over n ranks (layout_user.c:110-165):
// take the prime factors of n from the largest; each divides the direction
// whose block is longest (ties: the last such direction, unless an earlier
// one is already split and it is not); a factor that divides no block
// extent multiplies the longest direction's split without shrinking it.
static void hyper_split(const int len[4], int n, int nsq[4]) {
  static const int primes[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};
  int sq[4], extra[4];
  for (int i = 0; i < 4; i++) { sq[i] = len[i]; extra[i] = 1; nsq[i] = 1; }
  int k = (int)(sizeof primes / sizeof primes[0]) - 1;
  auto better = [&](int j, int i) {   // is direction i preferred to the current choice j?
    if (j < 0) return true;
    const long a = (long)extra[j] * sq[i], b = (long)extra[i] * sq[j];
    if (a > b) return true;
    return a == b && (nsq[j] == 1 || nsq[i] != 1);
  };
  while (n > 1) {
    while (k >= 0 && n % primes[k] != 0) --k;
    const int pf = k >= 0 ? primes[k] : n;
    int j = -1;
    for (int i = 0; i < 4; i++)
      if (sq[i] % pf == 0 && better(j, i)) j = i;
    n /= pf;
    if (j < 0) {
      for (int i = 0; i < 4; i++)
        if (better(j, i)) j = i;
      extra[j] *= pf;
    } else {
      sq[j] /= pf;
    }
    nsq[j] *= pf;
  }
}

// QMP's logical numbering: direction 0 varies fastest
static int rank_of(const int P[4], const int m[4]) { return m[0] + P[0] * (m[1] + P[1] * (m[2] + P[2] * m[3])); }
static void coords_of(const int P[4], int r, int m[4]) {
  for (int i = 0; i < 4; i++) { m[i] = r % P[i]; r /= P[i]; }
}

// node and node-local raw index of a global site for even blocks
// (layout_user.c:225-258)
static int node_of(const int L[4], const int P[4], const int x[4]) {
  int m[4];
  for (int i = 0; i < 4; i++) m[i] = (int)((long)x[i] * P[i] / L[i]);
  return rank_of(P, m);
}
static long node_index_of(const int L[4], const int P[4], const int x[4]) {
  long l = 0, vol = 1;
  int s = 0;
  for (int i = 0; i < 4; i++) {
    const int b = L[i] / P[i], m = (int)((long)x[i] * P[i] / L[i]);
    l = l * b + (x[i] - m * b);
    vol *= b;
    s += x[i];
  }
  return (s & 1) ? (l + vol) / 2 : l / 2;
}

// ---------------------------------------------------------------- state
struct Dd {
  int P[4], m[4], rank = 0, nranks = 1, mask = 0;
  int nbr[4][2];         // ranks of the -mu and +mu neighbours
  int fh[4];
  bool nccl = false;
  void *sraw[4] = {}, *sprod[4] = {}, *gup[4] = {}, *gdn[4] = {};
  size_t raw_cap[4] = {}, prod_cap[4] = {};
};

bool dd_active() {
  const Context &c = ctx();
  return c.dd && c.lat == 0;
}

void dd_refuse(const char *what) {
  if (ctx().dd) fail(QOP_FAIL, "%s is not available on a decomposed lattice", what);
}

// on a decomposed lattice only the fused int16 single-mass iteration has
// halo-reading kernels; every other sloppy form falls back to FP64
int sloppy_prec() {
  const Context &c = ctx();
  if (!c.dd) return c.opt.sloppy_prec;
  const Options &o = c.opt;
  return (o.sloppy_prec == 16 && o.half_format == 0 && o.fuse_update && (o.hop_kernel >= 20 || o.hop_kernel == -1)) ? 16 : 64;
}

void dd_allreduce(double *d, int n) {
  if (!dd_active()) return;
  Dd &dd = *ctx().dd;
  if (!dd.nccl || dd.nranks == 1) return;
  ncheck(g_nccl.AllReduce(d, d, (size_t)n, ncclDouble, ncclSum, g_comm.comm, ctx().s), "ncclAllReduce");
}

// sets up the decomposition for QOP_init; returns false (and prints why)
// when the layout is not usable; g becomes the local block's geometry
bool dd_setup(const QOP_layout_t *layout, Geom &g) {
  Context &c = ctx();
  int P[4] = {1, 1, 1, 1};
  const int *L = layout->latsize;
  if (layout->machdim > 0 && layout->machsize) {
    if (layout->machdim > 4) { fprintf(stderr, "QOP_init: machdim %d > 4\n", layout->machdim); return false; }
    for (int i = 0; i < layout->machdim; i++) P[i] = layout->machsize[i];
  } else if (g_comm.nranks > 1) {
    hyper_split(L, g_comm.nranks, P);
  }
  const int np = P[0] * P[1] * P[2] * P[3];
  if (np == 1 && !g_self_split) return true;
  if (np != g_comm.nranks) {
    fprintf(stderr, "QOP_init: %d blocks but %d processes in the communicator (QOPB_comm_init)\n", np,
            g_comm.nranks);
    return false;
  }
  Dd *d = new Dd();
  d->nranks = np;
  d->rank = g_comm.rank;
  d->nccl = g_comm.comm != nullptr;
  coords_of(P, d->rank, d->m);
  for (int i = 0; i < 4; i++) {
    d->P[i] = P[i];
    const int b = L[i] / P[i];
    if (L[i] % P[i] || b < 4 || (b & 1)) {
      fprintf(stderr, "QOP_init: extent %d split %d ways does not give even blocks of at least 4\n", L[i], P[i]);
      delete d;
      return false;
    }
    g.L[i] = b;
    g.O[i] = d->m[i] * b;
    g.GL[i] = L[i];
    if (P[i] > 1 || (g_self_split >> i & 1)) d->mask |= 1 << i;
    int mm[4] = {d->m[0], d->m[1], d->m[2], d->m[3]};
    mm[i] = (d->m[i] + P[i] - 1) % P[i];
    d->nbr[i][0] = rank_of(P, mm);
    mm[i] = (d->m[i] + 1) % P[i];
    d->nbr[i][1] = rank_of(P, mm);
  }
  g.V = (i64)g.L[0] * g.L[1] * g.L[2] * g.L[3];
  g.Vh = g.V / 2;
  c.dd = d;   // owned by the context from here: dd_free releases what was allocated
  try {
    for (int i = 0; i < 4; i++) {
      d->fh[i] = (int)(g.V / g.L[i] / 2);
      if (!(d->mask >> i & 1)) continue;
      // sized for FP64 and 16 links; one set serves both precisions
      d->raw_cap[i] = (size_t)dd_depth(16) * 3 * d->fh[i] * sizeof(double2);
      d->prod_cap[i] = (size_t)dd_nprod(16) * 3 * d->fh[i] * sizeof(double2);
      QCHECK(cudaMalloc(&d->sraw[i], d->raw_cap[i]));
      QCHECK(cudaMalloc(&d->gup[i], d->raw_cap[i]));
      QCHECK(cudaMalloc(&d->sprod[i], d->prod_cap[i]));
      QCHECK(cudaMalloc(&d->gdn[i], d->prod_cap[i]));
    }
  } catch (...) {
    dd_free();
    throw;
  }
  return true;
}

void dd_free() {
  Context &c = ctx();
  if (!c.dd) return;
  if (c.s) cudaStreamSynchronize(c.s);
  for (int i = 0; i < 4; i++) {
    cudaFree(c.dd->sraw[i]);
    cudaFree(c.dd->gup[i]);
    cudaFree(c.dd->sprod[i]);
    cudaFree(c.dd->gdn[i]);
  }
  delete c.dd;
  c.dd = nullptr;
}

// node of a global site and its node-local raw index (QOP_node_*_raw)
int dd_node_number(const int x[4]) {
  const Context &c = ctx();
  if (!c.dd) return 0;
  return node_of(c.lats[0].GL, c.dd->P, x);
}
long dd_node_index(const int x[4]) {
  const Context &c = ctx();
  const int one[4] = {1, 1, 1, 1};
  return node_index_of(c.lats[0].GL, c.dd ? c.dd->P : one, x);
}

// ---------------------------------------------------------------- halos
// one thread per (slab, face site): raw slabs s < depth hold the parity-q
// input at x_mu = s (for the -mu neighbour's up halo); product slab 0 holds
// -F_mu^+ psi at x_mu = L-1 and slab 1 + j holds -N_mu^+ psi at x_mu = L-1-j
// (for the +mu neighbour's down halo)
// one pack launch for every decomposed direction: entry j covers the
// threads [start[j], start[j+1]) of direction mu[j]
struct DdPackPlan {
  int n;
  int mu[4], fh[4];
  i64 start[5];
  void *sraw[4], *sprod[4];
};

static DdPackPlan dd_plan(const Dd &d, int nl) {
  DdPackPlan pl{};
  const int per = dd_depth(nl) + dd_nprod(nl);
  for (int mu = 0; mu < 4; mu++) {
    if (!(d.mask >> mu & 1)) continue;
    pl.mu[pl.n] = mu;
    pl.fh[pl.n] = d.fh[mu];
    pl.sraw[pl.n] = d.sraw[mu];
    pl.sprod[pl.n] = d.sprod[mu];
    pl.start[pl.n + 1] = pl.start[pl.n] + (i64)per * d.fh[mu];
    pl.n++;
  }
  return pl;
}

// the plan entry and slab coordinates of thread t (false past the end)
__device__ __forceinline__ bool dd_plan_entry(const DdPackPlan &pl, i64 t, int &j, int &s, int &fi) {
  if (t >= pl.start[pl.n]) return false;
  j = 0;
  while (j + 1 < pl.n && t >= pl.start[j + 1]) j++;
  const i64 l = t - pl.start[j];
  s = (int)(l / pl.fh[j]);
  fi = (int)(l % pl.fh[j]);
  return true;
}

template <typename T>
__global__ void k_dd_pack(const c2<T> *__restrict__ in, const c2<T> *__restrict__ lk, Geom g, int q, int nl,
                          DdPackPlan pl) {
  const int depth = dd_depth(nl);
  int j, s, fi;
  if (!dd_plan_entry(pl, blockIdx.x * (i64)blockDim.x + threadIdx.x, j, s, fi)) return;
  const int mu = pl.mu[j], fh = pl.fh[j];
  c2<T> *sraw = (c2<T> *)pl.sraw[j], *sprod = (c2<T> *)pl.sprod[j];
  int x[4];
  const int slot = dd_pack_site(g.L, mu, nl, q, s, fi, x);
  const i64 Vh = g.Vh;
  const int i = site_index(g, x[0], x[1], x[2], x[3]);
  const c2<T> v0 = in[i], v1 = in[Vh + i], v2 = in[2 * Vh + i];
  if (slot < 0) {
    c2<T> *o = sraw + (i64)s * 3 * fh + fi;
    o[0] = v0; o[fh] = v1; o[2 * fh] = v2;
    return;
  }
  const c2<T> *U = lk + (i64)slot * 9 * Vh + i;
  c2<T> *o = sprod + (i64)(s - depth) * 3 * fh + fi;
#pragma unroll
  for (int r = 0; r < 3; r++) {   // -(U^+ v)_r = -sum_c conj(U_cr) v_c
    c2<T> a = cconjmul<T>(U[r * Vh], v0);
    const c2<T> b = cconjmul<T>(U[(3 + r) * Vh], v1), e = cconjmul<T>(U[(6 + r) * Vh], v2);
    a = cadd<T>(cadd<T>(a, b), e);
    o[r * fh] = mk<T>(-a.x, -a.y);
  }
}

// moves the packed halos: every process posts the same sequence per
// direction (raw slabs to -mu, up halo from +mu, products to +mu, down halo
// from -mu), and NCCL matches the sends and receives between two processes
// in posting order.  rec_raw / rec_prod: bytes per face site and slab.
static void dd_exchange(Dd &d, int nl, size_t rec_raw, size_t rec_prod) {
  Context &c = ctx();
  const int depth = dd_depth(nl), np = dd_nprod(nl);
  if (d.nccl) {
    ncheck(g_nccl.GroupStart(), "ncclGroupStart");
    for (int mu = 0; mu < 4; mu++) {
      if (!(d.mask >> mu & 1)) continue;
      const size_t rb = (size_t)depth * d.fh[mu] * rec_raw, pb = (size_t)np * d.fh[mu] * rec_prod;
      ncheck(g_nccl.Send(d.sraw[mu], rb, ncclUint8, d.nbr[mu][0], g_comm.comm, c.s), "ncclSend");
      ncheck(g_nccl.Recv(d.gup[mu], rb, ncclUint8, d.nbr[mu][1], g_comm.comm, c.s), "ncclRecv");
      ncheck(g_nccl.Send(d.sprod[mu], pb, ncclUint8, d.nbr[mu][1], g_comm.comm, c.s), "ncclSend");
      ncheck(g_nccl.Recv(d.gdn[mu], pb, ncclUint8, d.nbr[mu][0], g_comm.comm, c.s), "ncclRecv");
    }
    ncheck(g_nccl.GroupEnd(), "ncclGroupEnd");
  } else {   // one process without a communicator: it is its own neighbour
    for (int mu = 0; mu < 4; mu++) {
      if (!(d.mask >> mu & 1)) continue;
      const size_t rb = (size_t)depth * d.fh[mu] * rec_raw, pb = (size_t)np * d.fh[mu] * rec_prod;
      QCHECK(cudaMemcpyAsync(d.gup[mu], d.sraw[mu], rb, cudaMemcpyDeviceToDevice, c.s));
      QCHECK(cudaMemcpyAsync(d.gdn[mu], d.sprod[mu], pb, cudaMemcpyDeviceToDevice, c.s));
    }
  }
}

template <typename T> DdGhost<T> dd_halo(FlaT<T> *f, const c2<T> *in, int q) {
  Context &c = ctx();
  Dd &d = *c.dd;
  const Geom &g = c.g;
  DdGhost<T> h{};
  h.mask = d.mask;
  const int nl = f->nlinks;
  const c2<T> *lk = f->d + (i64)q * nl * 9 * g.Vh;
  for (int mu = 0; mu < 4; mu++) {
    h.fh[mu] = d.fh[mu];
    h.up[mu] = (const c2<T> *)d.gup[mu];
    h.dn[mu] = (const c2<T> *)d.gdn[mu];
  }
  const DdPackPlan pl = dd_plan(d, nl);
  k_dd_pack<T><<<grid_for(pl.start[pl.n], 128), 128, 0, c.s>>>(in, lk, g, q, nl, pl);
  QLAUNCH();
  dd_exchange(d, nl, sizeof(c2<T>) * 3, sizeof(c2<T>) * 3);
  return h;
}

// int16 records: raw slabs copy the records; product slabs decode the
// record and the forward link from the solver's blocked int16 links (the
// same stored values the hop multiplies; 40 bytes per fat and 28 per
// reconstructed long link instead of 144 in FP64), apply -U^+ and store a
// new record
__device__ __forceinline__ void q16_link_decode(const unsigned char *lq, int nl, bool recon, float c_long, int k,
                                                i64 i, float2 U[9]) {
  const unsigned char *base = lq + (size_t)(i / QB) * q16_block_bytes(nl, recon) + q16_slot_off(k, recon);
  const int t = (int)(i % QB);
  const uint4 ua = reinterpret_cast<const uint4 *>(base)[t];
  U[0] = make_float2(u16_lo(ua.x), u16_hi(ua.x)); U[1] = make_float2(u16_lo(ua.y), u16_hi(ua.y));
  U[2] = make_float2(u16_lo(ua.z), u16_hi(ua.z)); U[3] = make_float2(u16_lo(ua.w), u16_hi(ua.w));
  float sc;
  if (recon && (k & 1)) {   // two rows / |c| and the det phase; row 2 = det conj(row0 x row1)
    const uint2 ub = reinterpret_cast<const uint2 *>(base + 16 * QB)[t];
    const float phase = reinterpret_cast<const float *>(base + 24 * QB)[t];
    U[4] = make_float2(u16_lo(ub.x), u16_hi(ub.x)); U[5] = make_float2(u16_lo(ub.y), u16_hi(ub.y));
    float sn, cs;
    __sincosf(phase, &sn, &cs);
    const float2 z = make_float2(cs * (1.0f / 32767.0f), sn * (1.0f / 32767.0f));
    const float2 c0 = csub<float>(cmul<float>(U[1], U[5]), cmul<float>(U[2], U[4]));
    const float2 c1 = csub<float>(cmul<float>(U[2], U[3]), cmul<float>(U[0], U[5]));
    const float2 c2 = csub<float>(cmul<float>(U[0], U[4]), cmul<float>(U[1], U[3]));
    U[6] = cmul<float>(z, make_float2(c0.x, -c0.y));
    U[7] = cmul<float>(z, make_float2(c1.x, -c1.y));
    U[8] = cmul<float>(z, make_float2(c2.x, -c2.y));
    sc = c_long * (1.0f / 32767.0f);
  } else {
    const uint4 ub = reinterpret_cast<const uint4 *>(base + 16 * QB)[t];
    const uint2 uc = reinterpret_cast<const uint2 *>(base + 32 * QB)[t];
    U[4] = make_float2(u16_lo(ub.x), u16_hi(ub.x)); U[5] = make_float2(u16_lo(ub.y), u16_hi(ub.y));
    U[6] = make_float2(u16_lo(ub.z), u16_hi(ub.z)); U[7] = make_float2(u16_lo(ub.w), u16_hi(ub.w));
    U[8] = make_float2(u16_lo(uc.x), u16_hi(uc.x));
    sc = __uint_as_float(uc.y) * (1.0f / 32767.0f);
  }
#pragma unroll
  for (int e = 0; e < 9; e++) U[e] = make_float2(U[e].x * sc, U[e].y * sc);
}

__global__ void k_dd_pack_q16(const uint4 *__restrict__ in, const unsigned char *__restrict__ lq, Geom g, int q,
                              int nl, bool recon, float c_long, DdPackPlan pl) {
  const int depth = dd_depth(nl);
  int j, s, fi;
  if (!dd_plan_entry(pl, blockIdx.x * (i64)blockDim.x + threadIdx.x, j, s, fi)) return;
  const int mu = pl.mu[j], fh = pl.fh[j];
  uint4 *sraw = (uint4 *)pl.sraw[j], *sprod = (uint4 *)pl.sprod[j];
  int x[4];
  const int slot = dd_pack_site(g.L, mu, nl, q, s, fi, x);
  const i64 Vh = g.Vh;
  const int i = site_index(g, x[0], x[1], x[2], x[3]);
  if (slot < 0) {
    sraw[(i64)s * fh + fi] = in[i];
    return;
  }
  float2 v[3], U[9];
  SpQ16::load(in, i, Vh, v);
  q16_link_decode(lq, nl, recon, c_long, slot, i, U);
  float2 o[3];
#pragma unroll
  for (int r = 0; r < 3; r++) {   // -(U^+ v)_r = -sum_c conj(U_cr) v_c
    float ax = 0.f, ay = 0.f;
#pragma unroll
    for (int cc = 0; cc < 3; cc++) {
      const float2 u = U[3 * cc + r];
      ax = fmaf(u.x, v[cc].x, fmaf(u.y, v[cc].y, ax));
      ay = fmaf(u.x, v[cc].y, fmaf(-u.y, v[cc].x, ay));
    }
    o[r] = make_float2(-ax, -ay);
  }
  SpQ16::store(sprod + (i64)(s - depth) * fh, fi, fh, o);
}

DdQ16Ghost dd_halo_q16(int nl, const unsigned char *lq, bool recon, float c_long, const uint4 *in, int q) {
  Context &c = ctx();
  Dd &d = *c.dd;
  const Geom &g = c.g;
  DdQ16Ghost h{};
  h.mask = d.mask;
  for (int mu = 0; mu < 4; mu++) {
    h.fh[mu] = d.fh[mu];
    h.up[mu] = (const uint4 *)d.gup[mu];
    h.dn[mu] = (const uint4 *)d.gdn[mu];
  }
  const DdPackPlan pl = dd_plan(d, nl);
  k_dd_pack_q16<<<grid_for(pl.start[pl.n], 128), 128, 0, c.s>>>(in, lq, g, q, nl, recon, c_long, pl);
  QLAUNCH();
  dd_exchange(d, nl, sizeof(uint4), sizeof(uint4));
  return h;
}

template DdGhost<float> dd_halo<float>(FlaT<float> *, const c2<float> *, int);
template DdGhost<double> dd_halo<double>(FlaT<double> *, const c2<double> *, int);

}  // namespace qopb

using namespace qopb;

#define DD_TRY try {
#define DD_CATCH(ret) } catch (Fail &e) { fprintf(stderr, "QOP error: %s\n", e.msg.c_str()); return ret; }

extern "C" {

int QOPB_comm_unique_id(unsigned char id[128]) {
  DD_TRY
  if (!id) return -1;
  nccl_load();
  ncclUniqueId u;
  ncheck(g_nccl.GetUniqueId(&u), "ncclGetUniqueId");
  memcpy(id, u.internal, sizeof u.internal);
  return 0;
  DD_CATCH(-1)
}

int QOPB_comm_init(const unsigned char id[128], int nranks, int rank) {
  DD_TRY
  if (!id || nranks < 1 || rank < 0 || rank >= nranks || g_comm.comm || ctx().inited) return -1;
  nccl_load();
  ensure_ready();
  ncclUniqueId u;
  memcpy(u.internal, id, sizeof u.internal);
  ncheck(g_nccl.CommInitRank(&g_comm.comm, nranks, u, rank), "ncclCommInitRank");
  g_comm.nranks = nranks;
  g_comm.rank = rank;
  return 0;
  DD_CATCH(-1)
}

int QOPB_comm_finalize(void) {
  if (ctx().inited) return -1;
  if (g_comm.comm) g_nccl.CommDestroy(g_comm.comm);
  g_comm = Comm();
  return 0;
}

int QOPB_dd_self_split(int mask) {
  if (ctx().inited || mask < 0 || mask > 15) return -1;
  g_self_split = mask;
  return 0;
}

int QOPB_layout_hyper(const int latsize[4], int nranks, int nsquares[4]) {
  if (!latsize || !nsquares || nranks < 1) return -1;
  hyper_split(latsize, nranks, nsquares);
  return 0;
}

int QOPB_layout_node_number(const int latsize[4], const int nsquares[4], const int coords[4]) {
  if (!latsize || !nsquares || !coords) return -1;
  return node_of(latsize, nsquares, coords);
}

long QOPB_layout_node_index(const int latsize[4], const int nsquares[4], const int coords[4]) {
  if (!latsize || !nsquares || !coords) return -1;
  return node_index_of(latsize, nsquares, coords);
}

int QOPB_layout_neighbors(const int nsquares[4], int rank, int nbr[8]) {
  if (!nsquares || !nbr) return -1;
  int m[4];
  coords_of(nsquares, rank, m);
  for (int i = 0; i < 4; i++) {
    int mm[4] = {m[0], m[1], m[2], m[3]};
    mm[i] = (m[i] + nsquares[i] - 1) % nsquares[i];
    nbr[2 * i] = rank_of(nsquares, mm);
    mm[i] = (m[i] + 1) % nsquares[i];
    nbr[2 * i + 1] = rank_of(nsquares, mm);
  }
  return 0;
}

int QOPB_dd_info(int nsquares[4], int coords[4], int local[4], int *mask) {
  const Context &c = ctx();
  if (!c.inited) return -1;
  for (int i = 0; i < 4; i++) {
    if (nsquares) nsquares[i] = c.dd ? c.dd->P[i] : 1;
    if (coords) coords[i] = c.dd ? c.dd->m[i] : 0;
    if (local) local[i] = c.lats[0].L[i];
  }
  if (mask) *mask = c.dd ? c.dd->mask : 0;
  return c.dd ? c.dd->rank : 0;
}

static bool dd_block_ok(const int local[4]) {
  if (!local) return false;
  for (int i = 0; i < 4; i++)
    if (local[i] < 4 || (local[i] & 1)) return false;
  return true;
}

int QOPB_dd_pack_site(const int local[4], int mu, int nlinks, int parity, int slab, int face, int x[4]) {
  if (!dd_block_ok(local) || !x || mu < 0 || mu > 3 || (nlinks != 8 && nlinks != 16) || (parity & ~1)) return -2;
  const long fh = (long)local[0] * local[1] * local[2] * local[3] / local[mu] / 2;
  if (slab < 0 || slab >= dd_depth(nlinks) + dd_nprod(nlinks) || face < 0 || face >= fh) return -2;
  return dd_pack_site(local, mu, nlinks, parity, slab, face, x);
}

int QOPB_dd_halo_ref(const int local[4], const int x[4], int mu, int disp, int *slab, int *face) {
  if (!dd_block_ok(local) || !x || !slab || !face || mu < 0 || mu > 3 ||
      (disp != 1 && disp != -1 && disp != 3 && disp != -3))
    return -1;
  for (int i = 0; i < 4; i++)
    if (x[i] < 0 || x[i] >= local[i]) return -1;
  const int y = x[mu] + disp;
  if ((unsigned)y < (unsigned)local[mu]) return 0;
  *slab = dd_halo_slab(local[mu], y, disp);
  *face = dd_face_index_L(local, x, mu);
  return y < 0 ? 2 : 1;
}

}  // extern "C"
