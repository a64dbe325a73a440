// solvers.cuh -- Krylov solvers and inverter drivers (solvers.cu, mixed.cu).
#pragma once
#include "qopb.h"
#include <vector>

namespace qopb {

// A = m^2 - D_eo,oe D_oe,eo on parity eo (QOP_asqtad_invert_d2 / _d2_norm2,
// lib/asqtad_invert_p.c:102-114)
template <typename T> struct LinOp {
  FlaT<T> *f;
  double mass;
  int eo;
  c2<T> *tmp;   // full-volume scratch; its opposite-parity half holds D_oe in
  void d2(c2<T> *out, const c2<T> *in) { Dslash<T>::ddagd(f, mass, out, in, eo, tmp, false); }
  double d2n(c2<T> *out, const c2<T> *in) { return Dslash<T>::ddagd(f, mass, out, in, eo, tmp, true); }
};

// full-volume FP64 vectors owned by a scope: freed on every way out of it,
// an allocation failure or a failed check included
struct ScopedVecs {
  std::vector<c2<double> *> v;
  ScopedVecs() = default;
  ScopedVecs(const ScopedVecs &) = delete;
  ScopedVecs &operator=(const ScopedVecs &) = delete;
  ~ScopedVecs() {
    for (c2<double> *q : v) dfree(q);
  }
  c2<double> *add() {
    v.reserve(v.size() + 1);
    v.push_back(dalloc<c2<double>>(vec_elems(ctx().g)));
    return v.back();
  }
};

template <typename T>
void cg(LinOp<T> &L, QOP_invert_arg_t *ia, QOP_resid_arg_t *ra, c2<T> *out, const c2<T> *in, c2<T> *p, int eo);
template <typename T>
void cgms(LinOp<T> &L, QOP_invert_arg_t *ia, QOP_resid_arg_t **ra, const double *shifts, int ns, c2<T> **out,
          const c2<T> *in, c2<T> *p, int eo);

// eigCG (cgtype 1): CG that accumulates low eigenvectors of A in the link
// handle and deflates the starting guess of later solves (eigcg.cu)
template <typename T>
void eigcg(LinOp<T> &L, QOP_invert_arg_t *ia, QOP_resid_arg_t *ra, c2<T> *out, const c2<T> *in, c2<T> *p, int eo,
           FlaT<T> *f);
// eigenvalues of the space stored for parity eo (at the mass of the last
// solve); copies up to max of them and returns how many are stored
template <typename T> int eigcg_values(FlaT<T> *f, int eo, double *l, int max);

template <typename T>
void invert(QOP_info_t *info, FlaT<T> *f, QOP_invert_arg_t *ia, QOP_resid_arg_t *ra, double mass, c2<T> *out,
            const c2<T> *in);
template <typename T>
void solve_multi(QOP_info_t *info, FlaT<T> *f, QOP_invert_arg_t *ia, QOP_resid_arg_t **ra, const double *masses,
                 c2<T> **out, c2<T> **in, int nsolve);
template <typename T>
void invert_multi(QOP_info_t *info, FlaT<T> *f, QOP_invert_arg_t *ia, QOP_resid_arg_t **ra[], double *masses[],
                  int nmass[], c2<T> **out[], c2<T> *in[], int nsrc);

// B200 mixed-precision inner solve (mixed.cu): multi-shift CG on A + shift_i
// with the Krylov iteration in reduced precision (FP32 or FP16 storage with
// FP32 arithmetic) and FP64 reliable updates of the true residual of the
// base system.  Returns false when the path is not applicable.
bool mixed_cgms(LinOp<double> &L, QOP_invert_arg_t *ia, QOP_resid_arg_t **ra, const double *shifts, int ns,
                c2<double> **out, const c2<double> *in, int eo, int prec);
// Independent systems (m_j^2 - D D) x_j = b_j on parity eo, solved
// together with int16 storage and one link stream per hop (batch.cu).  x_j
// holds the starting guess on entry and the solution on return; rsqmin_j is
// the target on |b_j - A_j x_j|^2 / |b_j|^2.  Returns per system its
// iteration count (hop pairs plus reliable updates) and the final FP64
// |r|^2 / |b|^2.
constexpr int BATCH_MAX = 16;
void run_batch(FlaT<double> *f, int eo, int n, const double *mass, c2<double> **x, c2<double> *const *b,
               const double *rsqmin, int max_iter, int *iters, double *final_rsq);

// makes s the library stream while in scope (nullptr: no change)
struct StreamScope {
  cudaStream_t old;
  explicit StreamScope(cudaStream_t s) : old(ctx().s) {
    if (s) ctx().s = s;
  }
  ~StreamScope() { ctx().s = old; }
  StreamScope(const StreamScope &) = delete;
  StreamScope &operator=(const StreamScope &) = delete;
};

// The solver of run_batch as a set of `cap` slots on one link handle and
// parity of the current lattice that systems enter and leave between steps
// (continuous batching): a system started while others are in flight joins
// their next hop launches; a finished slot can take a new system at once.
// Each system's iteration is independent of the others', so a system takes
// the same iterations and reaches the same solution alone or in a mix.
class BatchEngine {
 public:
  // own_stream: the engine's work runs on a stream of its own, so that the
  // chunks of several engines launched before any is collected overlap
  BatchEngine(FlaT<double> *f, int eo, int cap, bool own_stream = false);
  ~BatchEngine();
  BatchEngine(const BatchEngine &) = delete;
  BatchEngine &operator=(const BatchEngine &) = delete;
  // device bytes of an engine with cap slots on geometry g
  static size_t bytes(const Geom &g, int cap);
  int cap() const;
  int busy() const;       // slots holding a system (running or finished)
  int running() const;    // slots still iterating
  bool running(int s) const;   // slot s still iterating
  int free_slot() const;  // lowest free slot, or -1
  // start (m^2 - D D) x = b in free slot s; x (the starting guess, or zero
  // with x_zero) and b are FP64 device vectors the caller keeps until the
  // slot is released; rsqmin is the target on |b - A x|^2 / |b|^2
  void start(int s, c2<double> *x, const c2<double> *b, double mass, double rsqmin, int max_iter, bool x_zero);
  // one chunk of iterations of every running system, then their reliable
  // updates; returns the slots whose systems finished (x holds the solution)
  std::vector<int> step();
  // step() in two halves: launch() enqueues the chunk and returns at once;
  // collect() waits for it and serves the reliable updates.  Between the two
  // no slot may be started or released.
  void launch();
  std::vector<int> collect();
  cudaStream_t stream() const;   // the engine's stream (the library stream without own_stream)
  int iters(int s) const;         // hop pairs plus reliable updates
  double final_rsq(int s) const;  // FP64 |r|^2 / |b|^2
  void release(int s);
  // folds slot s's reduced-precision partial solution into its FP64 x
  // (between chunks), so that x is the system's current solution
  void fold(int s);

 private:
  struct Impl;
  Impl *d;
};
// several masses on one parity with prec_sloppy < 64: reduced-precision
// multi-shift CG per shared source, then per-solve refinement
void solve_multi_mixed(QOP_info_t *info, FlaT<double> *f, QOP_invert_arg_t *ia, QOP_resid_arg_t **ra,
                       const double *masses, c2<double> **out, c2<double> **in, int nsolve);

}  // namespace qopb
