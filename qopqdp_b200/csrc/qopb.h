// qopb.h -- internal declarations of the B200 asqtad/HISQ library.
//
// HBM layout (all fields checkerboarded, structure-of-arrays):
//   site index i in parity p: i = lex(x)/2 with lex = ((x0*L1+x1)*L2+x2)*L3+x3,
//   which is the reference raw index minus p*Vh (lib/layout_user.c:237-258),
//   so a raw parity half maps to a device parity block without reordering.
//   vector  : [parity][colour c][site i]            complex  (T2)
//   matrix  : [parity][element e=3a+b][site i]      complex
//   links   : [parity][slot k][element e][site i]   complex, slot k is the
//             reference's dbllinks order: 4mu+{fat fwd, long fwd, fat bck,
//             long bck}, shifts {+1,+3,-1,-3} along mu (16 slots; 8 without
//             Naik: 2mu+{fwd,bck}); links are stored times 1/2 as the reference
//             does (lib/asqtad_dslash_p.c:201-206).
// Consecutive threads take consecutive sites, so every link, mass-term and
// output access is a unit-stride coalesced load/store; neighbour gathers are
// unit stride within a row of x3 and hit L2 otherwise.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <stdexcept>
#include <vector>
#include "qop.h"
#include "qop_b200.h"

namespace qopb {

typedef long long i64;

// ---------------------------------------------------------------- errors
struct Fail {
  QOP_status_t status;
  std::string msg;
  Fail(QOP_status_t s, std::string m) : status(s), msg(std::move(m)) {}
};
void check_cuda(cudaError_t e, const char *what, const char *file, int line);
#define QCHECK(x) ::qopb::check_cuda((x), #x, __FILE__, __LINE__)
// every kernel launch is followed by QLAUNCH (or QLAUNCHN for n launches),
// which checks the launch and counts it (QOPB_launch_count)
void count_launches(int n);
#define QLAUNCHN(n) (::qopb::count_launches(n), ::qopb::check_cuda(cudaGetLastError(), "kernel launch", __FILE__, __LINE__))
#define QLAUNCH() QLAUNCHN(1)
[[noreturn]] void fail(QOP_status_t s, const char *fmt, ...);
// a NaN or Inf norm (of a source, a residual) ends the call with QOP_FAIL;
// the reference has no such check and would iterate on NaN
inline void need_finite(double v, const char *what) {
  if (!(v - v == 0.0)) fail(QOP_FAIL, "%s is not finite (%g): NaN or Inf in the input or the iteration", what, v);
}

// ---------------------------------------------------------------- geometry
struct Geom {
  int L[4];
  i64 V, Vh;
  // a decomposed lattice: this process holds the block of extents L at
  // global origin O (every O[mu] even) of the global lattice GL;
  // otherwise O = 0 and GL = L
  int O[4];
  int GL[4];
};
inline i64 global_vh(const Geom &g) { return (i64)g.GL[0] * g.GL[1] * g.GL[2] * g.GL[3] / 2; }

// ---------------------------------------------------------------- complex
template <typename T> struct Cx;
template <> struct Cx<float> { typedef float2 t; };
template <> struct Cx<double> { typedef double2 t; };
template <typename T> using c2 = typename Cx<T>::t;

template <typename T> __host__ __device__ inline c2<T> mk(T r, T i) { c2<T> z; z.x = r; z.y = i; return z; }
template <typename T> __host__ __device__ inline c2<T> cadd(c2<T> a, c2<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T> __host__ __device__ inline c2<T> csub(c2<T> a, c2<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <typename T> __host__ __device__ inline c2<T> cmul(c2<T> a, c2<T> b) {
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T> __host__ __device__ inline c2<T> cconjmul(c2<T> a, c2<T> b) {  // conj(a) b
  return mk<T>(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
template <typename T> __host__ __device__ inline c2<T> cscale(T s, c2<T> a) { return mk<T>(s * a.x, s * a.y); }
// acc += a*b
template <typename T> __host__ __device__ inline void cfma(c2<T> &acc, c2<T> a, c2<T> b) {
  acc.x += a.x * b.x - a.y * b.y;
  acc.y += a.x * b.y + a.y * b.x;
}

// host-side double complex used for solver scalars
struct dcx {
  double re, im;
};
inline dcx operator+(dcx a, dcx b) { return {a.re + b.re, a.im + b.im}; }
inline dcx operator-(dcx a, dcx b) { return {a.re - b.re, a.im - b.im}; }
inline dcx operator*(dcx a, dcx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline dcx operator*(double s, dcx a) { return {s * a.re, s * a.im}; }
inline dcx cdiv(dcx a, dcx b) {
  double d = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
inline double norm2(dcx a) { return a.re * a.re + a.im * a.im; }

// ---------------------------------------------------------------- context
struct Options {
  // QOP_asqtad_invert_set_opts (lib/asqtad_invert.c:69-113)
  int style = 1, nsvec = 8, nvec = 8, cgtype = 0;
  int eigcg_nev = 10, eigcg_m = 100, eigcg_numax = 200;
  // B200 additions: sloppy precision of the inner Krylov solve
  // (64 = exact reference algorithm in the handle's precision)
  int sloppy_prec = 64;
  int half_format = 0;           // 16-bit storage: 0 int16 fixed point, 1 IEEE FP16, 2 FP16 links
  double ru_delta = 0.3;         // reliable-update threshold on |r| (0.3-0.5 measured best)
  int chunk = 16;                // iterations launched per host check
  int hop_kernel = 25;           // int16 hop variant (mixed.cu launch_q16); 25 measured fastest; -1 autotuned
  int recon_long = 1;            // int16 long links as two rows + det phase when exact
  int batch_kernel = -1;         // batched int16 hop variant (batch.cu kBhop); -1: by the number of systems, -2: autotuned
  int multi_shift = 1;           // int16 multi-mass: 1 = sloppy multi-shift CG before the batched refinement (default), 0 = batched only
  double ms_stop = -1;           // multi-shift phase: a shifted system (not the lightest mass) stops at max(its rsqmin, ms_stop); -1: 1e-10 with int16 storage, else 0
  int fuse_update = 1;           // int16 hop variants 20-26: 1 = the second hop reduces for a fused x / r / p update
  int batch_tail = 1;            // batched solves: 1 = the last running system finishes in the one-system solver
  int pdl = 1;                   // fused int16 iteration: 1 = its kernels launched as programmatic dependents
  int serve_policy = 0;          // solve service: 0 = step every engine in turn, 1 = only the one with the oldest request
  double serve_hbm_mb = 0;       // solve service: device memory all engines together may hold (MB; 0 = free HBM less 2 GiB)
  int mbar_tries = 1 << 22;      // bounded mbarrier waits of the TMA-staged int16 hops: polls before MIX_ERROR
  // QOP_asqtad_force_set_opts (lib/asqtad_force.c:3-41)
  int force_fnmat_src_min = 2, force_veclength = 4;
  // QOP_hisq_force_set_opts (lib/hisq_force.c:4-52)
  int hisq_fnmat_src_min = 1, hisq_veclength = 4;
  double hisq_force_filter = 5e-5;
  // QOP_hisq_links_set_opts (lib/hisq_links.c:4-78)
  int want_deps = 0, want_aux = 1, reunit_allow_svd = 1, reunit_svd_only = 0;
  double reunit_svd_rel_error = 1e-8, reunit_svd_abs_error = 1e-8;
  int svd_values_info = 1, use_fat7_lepage = 0;
};

struct Context {
  int inited = 0;
  int verbosity = 0;
  int proflevel = 0;
  Geom g{};
  int device = 0;
  cudaStream_t s = nullptr;
  Options opt;
  // reduction scratch: per-block partials + completion counter + result
  double *d_part = nullptr;
  unsigned *d_count = nullptr;
  double *d_res = nullptr;
  double *h_res = nullptr;   // pinned
  int red_blocks = 0;
  size_t part_cap = 0;       // doubles in d_part
  // lattices: QOP_init defines lattice 0, QOPB_lattice_create adds more;
  // `g` is the geometry of the current one (QOPB_lattice_use)
  std::vector<Geom> lats;
  int lat = 0;
  struct Dd *dd = nullptr;   // domain decomposition of lattice 0 (dd.cu)
};
Context &ctx();
void require_init(const char *fn);
void ensure_ready();   // lazily creates stream and scratch on the current device

// stream-ordered device allocation, throws QOP_MEM_ERROR on failure
void *dmalloc(size_t bytes);
void dfree(void *p);
template <typename T> T *dalloc(i64 n) { return (T *)dmalloc(sizeof(T) * (size_t)n); }
void dzero(void *p, size_t bytes);
void sync();

int grid_for(i64 n, int block);

// ---------------------------------------------------------------- decomposition (dd.cu)
// true while lattice 0 is decomposed and current: hops exchange halos and
// reductions are summed over processes
bool dd_active();
// sums n doubles of a device buffer over the processes (stream ordered)
void dd_allreduce(double *d, int n);
// QOP_init: decomposes the lattice when the layout or the communicator asks
// for it (g becomes the local block); false when the layout is unusable
bool dd_setup(const QOP_layout_t *layout, Geom &g);
void dd_free();
int dd_node_number(const int x[4]);
long dd_node_index(const int x[4]);
// entry points without a decomposed form refuse with QOP_FAIL
void dd_refuse(const char *what);
// the sloppy precision the solvers use (on a decomposed lattice 16 only for
// the fused int16 single-mass iteration, whose kernels read halos; else 64)
int sloppy_prec();

// every handle remembers the lattice it was created on; entry points refuse
// handles of another lattice (their device arrays have another size)
void handle_register(const void *h);
void handle_forget(const void *h);
void handle_check(const void *h, const char *what);

// ---------------------------------------------------------------- handles
template <typename T> struct VecT {       // QOP_*_ColorVector
  c2<T> *d = nullptr;                     // [2][3][Vh]
};
template <typename T> struct GaugeT {     // QOP_*_GaugeField
  c2<T> *d = nullptr;                     // [4 mu][2][9][Vh]
  int *r0 = nullptr; QOP_Complex *bc = nullptr; int *signmask = nullptr;
};
struct SloppyLinks;                       // reduced-precision copies (mixed.cu)
template <typename T> struct FlaT {       // QOP_*_FermionLinksAsqtad
  int nlinks = 16;
  c2<T> *d = nullptr;                     // [2][nlinks][9][Vh], x 1/2, double stored
  SloppyLinks *sl = nullptr;
  void *shadow32 = nullptr;               // FlaT<float>* copy used by mixed solves
  void *eigcg = nullptr;                  // eigCG vector space (eigcg.cu), kept across solves
  void (*eigcg_free)(void *) = nullptr;
};
template <typename T> struct HisqT {      // QOP_*_FermionLinksHisq
  int n_naiks = 1;
  FlaT<T> *fn[QOP_MAX_NAIK] = {};
  FlaT<T> *fn_deps = nullptr;
  GaugeT<T> *U = nullptr, *V = nullptr, *W = nullptr;   // auxiliary links (want_aux)
};

inline i64 vec_elems(const Geom &g) { return 2 * 3 * g.Vh; }
inline i64 par_off(const Geom &g, int p) { return (i64)p * 3 * g.Vh; }

// subset helpers: a parity block of a vector is contiguous
struct Range { i64 off, n; };   // in complex elements
inline Range vrange(const Geom &g, int eo) {
  if (eo == QOP_EVEN) return {0, 3 * g.Vh};
  if (eo == QOP_ODD) return {3 * g.Vh, 3 * g.Vh};
  return {0, 6 * g.Vh};
}
inline int opp(int eo) { return eo == QOP_EVEN ? QOP_ODD : eo == QOP_ODD ? QOP_EVEN : QOP_EVENODD; }

// ---------------------------------------------------------------- BLAS (blas.cu)
template <typename T> struct Blas {
  static void zero(c2<T> *v, Range r);
  static void copy(c2<T> *d, const c2<T> *s, Range r);
  static void scale(c2<T> *d, double a, const c2<T> *s, Range r);                 // d = a s
  static void cscale(c2<T> *d, dcx a, const c2<T> *s, Range r);                   // d = a s
  static void axpy(c2<T> *y, double a, const c2<T> *x, Range r);                  // y += a x
  static void caxpy(c2<T> *y, dcx a, const c2<T> *x, Range r);                    // y += a x
  static void xpay(c2<T> *y, const c2<T> *x, double a, Range r);                  // y = x + a y
  static void axpby(c2<T> *z, double a, const c2<T> *x, double b, const c2<T> *y, Range r); // z = a x + b y
  static void caxpby(c2<T> *z, dcx a, const c2<T> *x, const c2<T> *y, Range r);   // z = a x + y
  static double norm2(const c2<T> *v, Range r);
  static double redot(const c2<T> *a, const c2<T> *b, Range r);
  static dcx cdot(const c2<T> *a, const c2<T> *b, Range r);                       // sum conj(a) b
  // x += a p ; r -= a Ap ; returns |r|^2
  static double cg_update(c2<T> *x, c2<T> *r, double a, const c2<T> *p, const c2<T> *Ap, Range q);
  // sum over sites of |r|^2/|x|^2 (1 where |x| = 0), single parity or both
  static double relnorm_sum(const c2<T> *r, const c2<T> *x, int eo);
};
// convert between precisions (d = s over range)
template <typename TD, typename TS> void convert(c2<TD> *d, const c2<TS> *s, Range r);

// ---------------------------------------------------------------- dslash (dslash.cu)
template <typename T> struct Dslash {
  // reference semantics of QOP_asqtad_dslash_qdp (lib/asqtad_dslash_p.c:1048-1092)
  static void apply(FlaT<T> *f, double mass, c2<T> *out, const c2<T> *in, int eo_out, int eo_in);
  // out_p = hop_p(in)  [+ epilogues]; parity p in {0,1}
  static void hop(FlaT<T> *f, c2<T> *out, const c2<T> *in, int p);
  static void dslash_dir(FlaT<T> *f, int dir, int fb, double wtfat, double wtlong,
                         c2<T> *out, const c2<T> *in, int eo_out);
  // ddagd (asqtad_dslash_p.c:1106-1138): out_eo = m^2 in - D_eo,oe D_oe,eo in;
  // tmp receives D_oe in on the opposite parity; returns |tmp|^2 + m^2 |in|^2
  static double ddagd(FlaT<T> *f, double mass, c2<T> *out, const c2<T> *in, int eo,
                      c2<T> *tmp, bool want_norm);
  // the same operator with caller-provided scratch: tmp_block is one parity
  // block ([3][Vh]), part/count/res the reduction partials, ticket and the
  // two sums; launches only, no allocation and no synchronisation
  static void ddagd_norm2_ws(FlaT<T> *f, double mass, c2<T> *out, const c2<T> *in, int eo, c2<T> *tmp_block,
                             double *part, unsigned *count, double *res);
};

// link construction (links.cu)
template <typename T> void double_store(FlaT<T> *f);
template <typename T> FlaT<T> *fla_from_fwd(const c2<T> *fat, const c2<T> *lng);   // fields [4][2][9][Vh], unscaled
template <typename TD, typename TS> FlaT<TD> *fla_convert(FlaT<TS> *src);
template <typename T> void fla_destroy(FlaT<T> *f);

void log0(int level, const char *fmt, ...);
double wtime();

}  // namespace qopb
