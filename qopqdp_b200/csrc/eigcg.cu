// eigcg.cu -- eigCG deflated CG (cgtype 1) for the EVENODD asqtad solve.
// Reference: lib/invert_eigcg_p.c:617-1068 (eigCG of Stathopoulos and
// Orginos, arXiv:0707.0131), lib/asqtad_invert_p.c:683-687, :767-770.
//
// While CG runs, the normalised residuals r_k/|r_k| are kept as a window of
// up to m Lanczos vectors v and the Lanczos matrix T is built from the CG
// coefficients (T_kk = 1/a_k + b_{k-1}/a_{k-1}, T_k,k-1 = -sqrt(b_{k-1})/a_{k-1}).
// When the window is full it is restarted with 2 nev vectors: the lowest nev
// Ritz vectors of T_m and of T_{m-1} (padded), orthonormalised and
// Rayleigh-Ritz rotated, plus the current residual.  At the end of a solve
// the lowest nev Ritz vectors of the last window join the stored space u,
// and the whole space is Rayleigh-Ritz rotated with the operator (eigen-
// values l).  Every later solve on the same links starts from the deflated
// guess x += sum_i u_i (u_i^+ r) / l_i.  Vectors stay on the device
// (full-volume arrays, operations on the solve parity); the small dense
// eigenproblems run on the host in FP64 (dense.cu).
//
// Differences from the reference, each a robustness fix that leaves the
// algorithm's steps alone:
//  - the handle keeps one space per solve parity.  The reference keeps one
//    space and assumes every solve runs on the same parity; the solve parity
//    follows the larger half of the source, and vectors of the other parity
//    are zero there (the reference's Gram-Schmidt then divides by zero).
//  - a solve at a new mass shifts the stored eigenvalues by the change of
//    m^2 (the eigenvectors of m^2 - D_pq D_qp do not depend on m).
//  - Gram-Schmidt drops vectors that lie numerically inside the span of the
//    earlier ones instead of normalising them.
//  - the window stops accumulating once the stored space plus a window of m
//    vectors would overrun numax (the reference writes past its array).
#include "solvers.cuh"
#include "dense.h"
#include <algorithm>
#include <cmath>
#include <vector>

namespace qopb {

namespace {

// out[j] = sum_i Y(i, j) in[i] for j < n2 (Y complex, row-major n1 x n2),
// elements [off, off + n) of every vector
template <typename T>
__global__ void k_rotate(c2<T> *const *out, const c2<T> *const *in, const double2 *Y, int n1, int n2, i64 off,
                         i64 n) {
  const i64 e = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (e >= n) return;
  constexpr int C = 8;
  for (int j0 = 0; j0 < n2; j0 += C) {
    double2 acc[C];
#pragma unroll
    for (int k = 0; k < C; k++) acc[k] = make_double2(0, 0);
    for (int i = 0; i < n1; i++) {
      const c2<T> v = in[i][off + e];
      const double2 x = make_double2((double)v.x, (double)v.y);
#pragma unroll
      for (int k = 0; k < C; k++)
        if (j0 + k < n2) {
          const double2 y = Y[(size_t)i * n2 + j0 + k];
          acc[k].x += y.x * x.x - y.y * x.y;
          acc[k].y += y.x * x.y + y.y * x.x;
        }
    }
#pragma unroll
    for (int k = 0; k < C; k++)
      if (j0 + k < n2) out[j0 + k][off + e] = mk<T>((T)acc[k].x, (T)acc[k].y);
  }
}

}  // namespace

template <typename T> struct DVec {   // scoped full-volume device vector
  c2<T> *p;
  DVec() { p = dalloc<c2<T>>(vec_elems(ctx().g)); dzero(p, sizeof(c2<T>) * vec_elems(ctx().g)); }
  ~DVec() { dfree(p); }
  operator c2<T> *() const { return p; }
};

template <typename T> struct EigcgState {
  int nev = 0, m = 0, numax = 0;
  int nu = 0, nv = 0, nn = 0, addvecs = 1;
  double mass = 0;              // mass the eigenvalues l belong to
  std::vector<c2<T> *> u;       // numax full-volume vectors (u[0..nu) eigenvectors, then the window)
  std::vector<double> l;        // Rayleigh-Ritz eigenvalues of u[0..nu)
  ~EigcgState() {
    for (auto *p : u) dfree(p);
  }
};

// one space per parity: eigenvectors of m^2 - H_pq H_qp on parity p
template <typename T> struct EigcgSpaces {
  EigcgState<T> *s[2] = {nullptr, nullptr};
  ~EigcgSpaces() { delete s[0]; delete s[1]; }
};

template <typename T> static void eigcg_free(void *s) { delete reinterpret_cast<EigcgSpaces<T> *>(s); }

// v[0..n2) <- v[0..n1) Y  (complex n1 x n2, n2 <= n1)
template <typename T>
static void rotate(c2<T> **v, int n1, int n2, const std::vector<zc> &Y, Range q) {
  Context &c = ctx();
  std::vector<c2<T> *> tmp(n2);
  for (int j = 0; j < n2; j++) tmp[j] = dalloc<c2<T>>(vec_elems(c.g));
  std::vector<double2> hy((size_t)n1 * n2);
  for (size_t k = 0; k < hy.size(); k++) hy[k] = make_double2(Y[k].real(), Y[k].imag());
  double2 *dy = dalloc<double2>((i64)hy.size());
  c2<T> **din = dalloc<c2<T> *>(n1), **dout = dalloc<c2<T> *>(n2);
  QCHECK(cudaMemcpyAsync(dy, hy.data(), sizeof(double2) * hy.size(), cudaMemcpyHostToDevice, c.s));
  QCHECK(cudaMemcpyAsync(din, v, sizeof(void *) * n1, cudaMemcpyHostToDevice, c.s));
  QCHECK(cudaMemcpyAsync(dout, tmp.data(), sizeof(void *) * n2, cudaMemcpyHostToDevice, c.s));
  k_rotate<T><<<grid_for(q.n, 128), 128, 0, c.s>>>(dout, din, dy, n1, n2, q.off, q.n);
  QLAUNCH();
  for (int j = 0; j < n2; j++) {
    Blas<T>::copy(v[j], tmp[j], q);
    dfree(tmp[j]);
  }
  dfree(dy); dfree(din); dfree(dout);
}

template <typename T>
static void rotate_real(c2<T> **v, int n1, int n2, const std::vector<double> &Y, int ld, Range q) {
  std::vector<zc> Z((size_t)n1 * n2);
  for (int i = 0; i < n1; i++)
    for (int j = 0; j < n2; j++) Z[(size_t)i * n2 + j] = Y[(size_t)i * ld + j];
  rotate<T>(v, n1, n2, Z, q);
}

// Gram-Schmidt of v[i0..i0+n) against v[0..i) in turn (invert_eigcg_p.c:209-221).
// A vector left with less than 1e-24 of its norm (numerically inside the
// span of the earlier ones; the reference would divide by ~0 there) is
// dropped: its buffer moves behind the kept ones.  Returns the kept count.
template <typename T>
static int orthonormalize(c2<T> **v, int i0, int n, Range q) {
  typedef Blas<T> B;
  int end = i0 + n;
  for (int i = i0; i < end;) {
    const double n0 = B::norm2(v[i], q);
    for (int j = 0; j < i; j++) {
      const dcx z = B::cdot(v[j], v[i], q);
      B::caxpy(v[i], dcx{-z.re, -z.im}, v[j], q);
    }
    const double n1 = B::norm2(v[i], q);
    if (!(n1 > 1e-24 * n0) || !std::isfinite(n1)) {
      c2<T> *d = v[i];
      for (int k = i; k < end - 1; k++) v[k] = v[k + 1];
      v[--end] = d;
      continue;
    }
    B::scale(v[i], 1.0 / std::sqrt(n1), v[i], q);
    i++;
  }
  return end - i0;
}

// Rayleigh-Ritz of u[0..nu+nv): u[nu..) orthonormalised, the first nu
// assumed to be eigenvectors with eigenvalues l (:223-309).  Returns the
// size of the rotated space (nu plus the independent new vectors).
template <typename T>
static int rayleigh_ritz(LinOp<T> &L, c2<T> **u, std::vector<double> &l, int nu, int nv, c2<T> *p, c2<T> *Mp,
                         Range q) {
  typedef Blas<T> B;
  if (nu + nv <= 0) return 0;
  const int n = nu + orthonormalize<T>(u, nu, nv, q);
  if (n <= 0) return 0;
  std::vector<zc> mm((size_t)n * n, zc(0, 0)), tt;
  for (int i = 0; i < nu; i++) mm[(size_t)i * n + i] = l[i];
  for (int j = nu; j < n; j++) {
    B::copy(p, u[j], q);
    L.d2(Mp, p);
    for (int i = 0; i <= j; i++) {
      const dcx z = B::cdot(u[i], Mp, q);
      mm[(size_t)i * n + j] = zc(z.re, z.im);
      mm[(size_t)j * n + i] = zc(z.re, -z.im);
    }
    mm[(size_t)j * n + j] = zc(mm[(size_t)j * n + j].real(), 0.0);
  }
  std::vector<double> vv;
  herm_eig(n, mm, vv, tt);
  rotate<T>(u, n, n, tt, q);
  for (int i = 0; i < n; i++) l[i] = vv[i];
  log0(QOP_VERB_MED, "eigCG: rr: n %d ev[0] %g ev[%d] %g\n", n, vv[0], n - 1, vv[n - 1]);
  if (ctx().verbosity >= QOP_VERB_MED) {   // residuals |A u - l u| (:284-312)
    int ngood = 0;
    for (int i = 0; i < n; i++) {
      B::copy(p, u[i], q);
      L.d2(Mp, p);
      B::axpy(Mp, -l[i], u[i], q);
      const double rr = std::sqrt(B::norm2(Mp, q));
      if (rr <= 1e-4 && ngood == i) ngood++;
      if (i < 2 || i == n - 1) log0(QOP_VERB_MED, "eigCG: ev[%d] %g resid %g\n", i, l[i], rr);
    }
    log0(QOP_VERB_MED, "eigCG: ngood %d of %d\n", ngood, n);
  }
  return n;
}

// A new mass shifts every stored eigenvalue by the change of m^2 (the
// operator is m^2 - H_pq H_qp; its eigenvectors do not depend on m).
template <typename T>
static void shift_mass(EigcgState<T> *E, double mass) {
  if (E->mass != mass)
    for (int i = 0; i < E->nu; i++) E->l[i] += mass * mass - E->mass * E->mass;
  E->mass = mass;
}

// dense window algebra (:418-526): T (m x m), TD eigenvalues, TB eigenvectors,
// Y (m x 2 nev), all row-major with leading dimension m (Y: 2 nev)
struct Window {
  int m, nev;
  std::vector<double> t, td, tb, y;
  Window(int m_, int nev_) : m(m_), nev(nev_), t((size_t)m_ * m_, 0.0), td(m_), tb((size_t)m_ * m_), y((size_t)m_ * 2 * nev_) {}
  double &T(int i, int j) { return t[(size_t)i * m + j]; }
  double &TB(int i, int j) { return tb[(size_t)i * m + j]; }
  double &Y(int i, int j) { return y[(size_t)i * 2 * nev + j]; }
  // all eigenpairs of T[0:n, 0:n] into td, tb
  void diag(int n) {
    std::vector<double> a((size_t)n * n), w, z;
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) a[(size_t)i * n + j] = T(i, j);
    sym_eig(n, a, w, z);
    for (int i = 0; i < n; i++) {
      td[i] = w[i];
      for (int j = 0; j < n; j++) TB(i, j) = z[(size_t)i * n + j];
    }
  }
  // Y[0:nvv, noff:noff+k] = TB[0:nvv, 0:k], zero below; for noff > 0 the new
  // columns are orthonormalised against the first noff, and TB[0:n, 0:noff+k]
  // becomes Y rotated by the eigenvectors of Y^T T Y (td its eigenvalues)
  void set_y(int noff, int k, int nvv, int n) {
    for (int i = 0; i < n; i++)
      for (int j = 0; j < k; j++) Y(i, noff + j) = i < nvv ? TB(i, j) : 0.0;
    if (!noff) return;
    const int w = noff + k;
    for (int c = noff; c < w; c++) {   // dorthocols: against the earlier columns
      for (int c2i = 0; c2i < c; c2i++) {
        double s = 0;
        for (int i = 0; i < n; i++) s += Y(i, c2i) * Y(i, c);
        for (int i = 0; i < n; i++) Y(i, c) -= s * Y(i, c2i);
      }
      double nr = 0;
      for (int i = 0; i < n; i++) nr += Y(i, c) * Y(i, c);
      nr = 1.0 / std::sqrt(nr);
      for (int i = 0; i < n; i++) Y(i, c) *= nr;
    }
    std::vector<double> ty((size_t)n * w, 0.0), h((size_t)w * w, 0.0), hw, hz;
    for (int i = 0; i < n; i++)
      for (int j = 0; j < w; j++) {
        double s = 0;
        for (int k2 = 0; k2 < n; k2++) s += T(i, k2) * Y(k2, j);
        ty[(size_t)i * w + j] = s;
      }
    for (int a = 0; a < w; a++)
      for (int b = 0; b < w; b++) {
        double s = 0;
        for (int i = 0; i < n; i++) s += Y(i, a) * ty[(size_t)i * w + b];
        h[(size_t)a * w + b] = s;
      }
    sym_eig(w, h, hw, hz);
    for (int j = 0; j < w; j++) td[j] = hw[j];
    for (int i = 0; i < n; i++)
      for (int j = 0; j < w; j++) {
        double s = 0;
        for (int a = 0; a < w; a++) s += Y(i, a) * hz[(size_t)a * w + j];
        TB(i, j) = s;
      }
  }
};

template <typename T>
void eigcg(LinOp<T> &L, QOP_invert_arg_t *ia, QOP_resid_arg_t *ra, c2<T> *out, const c2<T> *in, c2<T> *p, int eo,
           FlaT<T> *f) {
  typedef Blas<T> B;
  Context &c = ctx();
  const Range q = vrange(c.g, eo);
  const Options &o = c.opt;
  EigcgSpaces<T> *S = reinterpret_cast<EigcgSpaces<T> *>(f->eigcg);
  if (!S) {
    S = new EigcgSpaces<T>();
    f->eigcg = S;
    f->eigcg_free = eigcg_free<T>;
  }
  EigcgState<T> *&E = S->s[eo == QOP_ODD ? 1 : 0];
  if (E && (E->numax != o.eigcg_numax)) {   // space size changed: start afresh
    delete E;
    E = nullptr;
  }
  if (!E) {
    E = new EigcgState<T>();
    E->numax = o.eigcg_numax;
    E->mass = L.mass;
    E->u.assign(E->numax, nullptr);
    for (auto &v : E->u) {
      v = dalloc<c2<T>>(vec_elems(c.g));
      dzero(v, sizeof(c2<T>) * vec_elems(c.g));
    }
    E->l.assign(E->numax, 0.0);
  }
  E->nev = o.eigcg_nev;
  E->m = o.eigcg_m;
  const int nev = E->nev, m = E->m, numax = E->numax;
  if (nev < 1 || m < 2 * nev + 2 || numax < m + nev) fail(QOP_FAIL, "eigCG: need m >= 2 nev + 2 and numax >= m + nev");
  shift_mass<T>(E, L.mass);
  int nu = E->nu, nv = E->nv, nn = E->nn, addvecs = E->addvecs;
  c2<T> **u = E->u.data();
  std::vector<double> &l = E->l;
  DVec<T> r, Mp;
  const int max_it = ia->max_iter;
  int max_restarts = ia->max_restarts < 0 ? 5 : ia->max_restarts;
  ra->final_rsq = ra->final_rel = 0;
  ra->final_iter = ra->final_restart = 0;
  const double insq = B::norm2(in, q);
  if (insq == 0.) { B::zero(out, q); return; }
  const double rsqstop = ra->rsqmin * insq;
  double rsq = 0, oldrsq = 0, relnorm = 1, a = 0, a0 = 0, b = 0;
  int total = 0, nrestart = -1;
  auto done = [&]() {
    return ((rsqstop <= 0 || rsq < rsqstop) && (ra->relmin <= 0 || relnorm < ra->relmin)) || total >= max_it;
  };
  auto true_resid = [&]() {
    B::copy(p, out, q);
    L.d2(Mp, p);
    total++;
    B::axpby(r, 1.0, in, -1.0, Mp, q);
    rsq = B::norm2(r, q);
    if (ra->relmin > 0) relnorm = Blas<T>::relnorm_sum(r, out, eo) / (double)global_vh(ctx().g);
  };
  Window W(m, nev);
  c2<T> **v = nullptr;
  auto setv = [&]() {   // v[nv] = r / |r|
    B::scale(v[nv], 1.0 / std::sqrt(rsq), r, q);
    nv++;
  };
  do {
    true_resid();
    log0(QOP_VERB_LOW, "eigCG: (re)start: iter %d rsq = %g rel = %g\n", total, rsq, relnorm);
    if (done()) break;
    if (addvecs && nn >= m) {   // :735-755
      int nr = numax - 2 * m - 1;
      if (nr >= nu) nr = nu - 2;
      if (nr < 0) nr = 0;
      const double oldl = nu == 0 ? 9999 : l[nr];
      nu = rayleigh_ritz<T>(L, u, l, nu, nn, p, Mp, q);
      nn = 0;
      const double delta = std::fabs(2 * (oldl - l[nr]) / (oldl + l[nr]));
      if (delta < 1e-4) addvecs = 0;
      else if (nu > numax - 2 * m) nu = numax - 2 * m;
    }
    if (nu > 0) {   // deflated start (:322-341, :757-777)
      B::zero(p, q);
      for (int i = 0; i < nu; i++) {
        const dcx z = B::cdot(u[i], r, q);
        B::caxpy(p, dcx{z.re / l[i], z.im / l[i]}, u[i], q);
      }
      B::axpy(out, 1.0, p, q);
      true_resid();
      log0(QOP_VERB_LOW, "eigCG: proj u: iter %d rsq = %g rel = %g\n", total, rsq, relnorm);
      if (done()) break;
    }
    // the window needs m + 1 free slots beyond the stored space
    if (addvecs && nu + nn + m + 1 > numax) addvecs = 0;
    if (addvecs) {
      v = u + nu + nn;
      std::fill(W.t.begin(), W.t.end(), 0.0);
    }
    B::copy(p, r, q);
    while (true) {
      L.d2(Mp, p);
      total++;
      const double pkp = B::redot(p, Mp, q);
      if (pkp <= 0) break;
      a0 = a;
      a = rsq / pkp;
      if (addvecs) {   // :915-949
        if (nv == 0) {
          W.T(0, 0) = 1.0 / a;
          setv();
        } else if (nv < m) {
          W.T(nv, nv) = 1.0 / a + b / a0;
          W.T(nv, nv - 1) = W.T(nv - 1, nv) = -std::sqrt(b) / a0;
          setv();
        } else {
          // thick restart: lowest nev Ritz vectors of T_m and of T_{m-1}
          W.diag(nv);
          W.set_y(0, nev, nv, nv);
          W.diag(nv - 1);
          W.set_y(nev, nev, nv - 1, nv);
          rotate_real<T>(v, nv, 2 * nev, W.tb, m, q);
          // reset T with the new residual as vector 2 nev (:551-596)
          nv = 2 * nev;
          setv();
          std::fill(W.t.begin(), W.t.end(), 0.0);
          c2<T> *sp = dalloc<c2<T>>(vec_elems(ctx().g)), *sMp = dalloc<c2<T>>(vec_elems(ctx().g));
          B::copy(sp, p, q);
          B::copy(sMp, Mp, q);
          B::copy(p, v[nv - 1], q);
          L.d2(Mp, p);
          for (int i = 0; i < nv - 1; i++) {
            const double rr = B::redot(v[i], Mp, q);
            W.T(i, nv - 1) = W.T(nv - 1, i) = rr;
            W.T(i, i) = W.td[i];
          }
          W.T(nv - 1, nv - 1) = 1.0 / a + b / a0;
          B::copy(p, sp, q);
          B::copy(Mp, sMp, q);
          dfree(sp);
          dfree(sMp);
        }
      }
      oldrsq = rsq;
      rsq = B::cg_update(out, r, a, p, Mp, q);
      if (ra->relmin > 0) relnorm = Blas<T>::relnorm_sum(r, out, eo) / (double)global_vh(ctx().g);
      log0(QOP_VERB_HI, "eigCG: iter %d rsq = %g rel = %g\n", total, rsq, relnorm);
      if (done()) break;
      b = rsq / oldrsq;
      B::xpay(p, r, b, q);
    }
    if (addvecs) {   // :1000-1022: lowest nev Ritz vectors of the last window
      if (nv > nev) {
        const int k = orthonormalize<T>(v, 0, nv, q), ne = std::min(nev, k);
        for (int j = 0; j < k; j++) {   // T = v^+ A v, real part
          B::copy(p, v[j], q);
          L.d2(Mp, p);
          for (int i = 0; i < k; i++) W.T(i, j) = B::redot(v[i], Mp, q);
        }
        if (ne > 0) {
          W.diag(k);
          W.set_y(0, ne, k, k);
          rotate_real<T>(v, k, ne, W.tb, m, q);
          nn += ne;
        }
      }
      nv = 0;
    }
    nrestart++;
  } while (total < max_it && nrestart < max_restarts);
  if (addvecs) {   // :1030-1036
    nu = rayleigh_ritz<T>(L, u, l, 0, nu + nn + nv, p, Mp, q);
    nn = nv = 0;
  }
  E->nu = nu;
  E->nv = nv;
  E->nn = nn;
  E->addvecs = addvecs;
  ra->final_rsq = rsq / insq;
  ra->final_rel = relnorm;
  ra->final_iter = total;
  ra->final_restart = nrestart;
}

template <typename T> int eigcg_values(FlaT<T> *f, int eo, double *l, int max) {
  const EigcgSpaces<T> *S = reinterpret_cast<const EigcgSpaces<T> *>(f->eigcg);
  const EigcgState<T> *E = S ? S->s[eo == QOP_ODD ? 1 : 0] : nullptr;
  if (!E) return 0;
  for (int i = 0; i < E->nu && i < max; i++) l[i] = E->l[i];
  return E->nu;
}

template int eigcg_values<float>(FlaT<float> *, int, double *, int);
template int eigcg_values<double>(FlaT<double> *, int, double *, int);
template void eigcg<float>(LinOp<float> &, QOP_invert_arg_t *, QOP_resid_arg_t *, c2<float> *, const c2<float> *,
                           c2<float> *, int, FlaT<float> *);
template void eigcg<double>(LinOp<double> &, QOP_invert_arg_t *, QOP_resid_arg_t *, c2<double> *,
                            const c2<double> *, c2<double> *, int, FlaT<double> *);

}  // namespace qopb
