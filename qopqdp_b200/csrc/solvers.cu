// solvers.cu -- QOPQDP's Krylov solvers and asqtad inverter drivers on the
// device.  Control flow, stopping rules and scalar recurrences (FP64) follow
// the reference line by line; every vector operation is a device kernel.
// Reference: lib/invert_cg_p.c:1-128 (CG), :130-402 (multi-shift CG),
// lib/invert_utilities_p.c:1-40 (Fermilab relative norm),
// lib/asqtad_invert_p.c:80-100 (project/reconstruct), :246-330 (refine),
// :332-647 (solve_multi), :649-851 (invert), :878-1059 (invert_multi).
#include "solvers.cuh"
#include <memory>
#include "fields.cuh"
#include <vector>
#include <cmath>
#include <type_traits>

namespace qopb {

template <typename T> struct Tmp {   // scoped full-volume device vector
  c2<T> *p;
  Tmp() { p = dalloc<c2<T>>(vec_elems(ctx().g)); dzero(p, sizeof(c2<T>) * vec_elems(ctx().g)); }
  ~Tmp() { dfree(p); }
  operator c2<T> *() const { return p; }
};

template <typename T> static double relnorm2(const c2<T> *r, const c2<T> *x, int eo) {
  const Geom &g = ctx().g;
  double n = eo == QOP_EVENODD ? 2.0 * global_vh(g) : (double)global_vh(g);
  return Blas<T>::relnorm_sum(r, x, eo) / n;
}

// ---------------------------------------------------------------- CG
template <typename T>
void cg(LinOp<T> &L, QOP_invert_arg_t *ia, QOP_resid_arg_t *ra, c2<T> *out, const c2<T> *in, c2<T> *p, int eo) {
  typedef Blas<T> B;
  const Range q = vrange(ctx().g, eo);
  int iteration = 0, total = 0, nrestart = -1;
  const int restart_it = ia->restart, max_it = ia->max_iter;
  int max_restarts = ia->max_restarts;
  if (max_restarts < 0) max_restarts = 5;
  ra->final_rsq = 0; ra->final_rel = 0; ra->final_iter = 0; ra->final_restart = 0;
  double insq = B::norm2(in, q);
  need_finite(insq, "CG: source norm");
  if (insq == 0.) { B::zero(out, q); return; }
  Tmp<T> r, Mp;
  double rsqstop = ra->rsqmin * insq, rsq = 0, oldrsq = 0, relnorm = 1;
  log0(QOP_VERB_LOW, "CG: rsqmin = %g relmin = %g\nCG: rsqstop = %g\n", ra->rsqmin, ra->relmin, rsqstop);
  while (true) {
    if (total == 0 || iteration >= restart_it || total >= max_it || rsq < rsqstop || relnorm < ra->relmin) {
      if (total >= max_it || nrestart >= max_restarts) break;
      nrestart++;
      B::copy(p, out, q);
      L.d2(Mp, p);
      iteration = 1; total++;
      B::axpby(r, 1.0, in, -1.0, Mp, q);
      rsq = B::norm2(r, q);
      need_finite(rsq, "CG: true residual norm");
      if (ra->relmin > 0) relnorm = relnorm2<T>(r, out, eo);
      log0(QOP_VERB_LOW, "CG: (re)start: iter %i rsq = %g rel = %g\n", total, rsq, relnorm);
      if (rsq < rsqstop || relnorm < ra->relmin || total >= max_it) break;
      B::copy(p, r, q);
    } else {
      double b = rsq / oldrsq;
      B::xpay(p, r, b, q);
    }
    oldrsq = rsq;
    L.d2(Mp, p);
    iteration++; total++;
    double pkp = B::redot(p, Mp, q);
    need_finite(pkp, "CG: <p, A p>");
    if (pkp <= 0) break;
    double a = rsq / pkp;
    rsq = B::cg_update(out, r, a, p, Mp, q);
    if (ra->relmin > 0) relnorm = relnorm2<T>(r, out, eo);
    log0(QOP_VERB_HI, "CG: iter %i rsq = %g rel = %g\n", total, rsq, relnorm);
  }
  ra->final_rsq = rsq / insq;
  ra->final_rel = relnorm;
  ra->final_iter = total;
  ra->final_restart = nrestart;
}

// ---------------------------------------------------------------- multi-shift CG
template <typename T>
void cgms(LinOp<T> &L, QOP_invert_arg_t *ia, QOP_resid_arg_t **ra, const double *shifts, int ns, c2<T> **out,
          const c2<T> *in, c2<T> *p, int eo) {
  typedef Blas<T> B;
  const Range q = vrange(ctx().g, eo);
  std::vector<double> a(ns, 0), b(ns, 0), bo(ns, -1), z(ns, 1), zo(ns, 1), zn(ns, 1);
  double insq = B::norm2(in, q);
  need_finite(insq, "CGMS: source norm");
  if (insq == 0.) {
    for (int i = 0; i < ns; i++) {
      B::zero(out[i], q);
      ra[i]->final_rsq = ra[i]->final_rel = 0; ra[i]->final_iter = ra[i]->final_restart = 0;
    }
    return;
  }
  int imin = 0, irsq = 0, irel = 0, iteration = 0;
  for (int i = 1; i < ns; i++) {
    if (shifts[i] < shifts[imin]) imin = i;
    if (ra[i]->rsqmin >= ra[irsq]->rsqmin) irsq = i;
    if (ra[i]->relmin > ra[irel]->relmin) irel = i;
  }
  const double rsqstop = ra[irsq]->rsqmin * insq, relstop = ra[irel]->relmin;
  Tmp<T> r, Mp, y, Ay, ry;
  std::vector<std::unique_ptr<Tmp<T>>> own;
  std::vector<c2<T> *> pm(ns);
  B::copy(r, in, q);
  for (int i = 0; i < ns; i++) {
    if (i == imin) pm[i] = p;
    else { own.emplace_back(new Tmp<T>()); pm[i] = *own.back(); }
    B::zero(out[i], q);
    B::copy(pm[i], r, q);
  }
  log0(QOP_VERB_MED, "CGMS: rsqmin: %g  relmin: %g  in2: %g  rsqstop: %g\n", ra[irsq]->rsqmin, relstop, insq, rsqstop);
  double rsq = insq, oldrsq, relnorm = 1, trueRsqFac = 1, trueRelFac = 1, yAy = 0;
  const int rsqCheckInterval = 100, relCheckInterval = 100;
  int nextRsqCheck = rsqCheckInterval, nextRelCheck = relCheckInterval;
  B::copy(ry, in, q);
  while (true) {
    oldrsq = rsq;
    double pkp = L.d2n(Mp, p);
    iteration++;
    need_finite(pkp, "CGMS: <p, A p>");
    if (pkp <= 0) break;
    b[imin] = rsq / pkp;
    rsq = B::cg_update(out[imin], r, b[imin], p, Mp, q);
    zn[imin] = 1;
    for (int i = 0; i < ns; i++) {
      if (i == imin) continue;
      zn[i] = z[i] * zo[i] * bo[imin];
      double c1 = b[imin] * a[imin] * (zo[i] - z[i]);
      c1 += zo[i] * bo[imin] * (1 + shifts[i] * b[imin]);
      if (c1 != 0.0) zn[i] /= c1; else zn[i] = 0;
      if (z[i] != 0.0) b[i] = b[imin] * zn[i] / z[i]; else zn[i] = b[i] = 0;
    }
    for (int i = 0; i < ns; i++)
      if (i != imin) B::axpy(out[i], b[i], pm[i], q);
    double rsqc = zn[irsq] * zn[irsq] * rsq;
    if (relstop > 0) relnorm = zn[irel] * zn[irel] * relnorm2<T>(r, out[irel], eo);
    log0(QOP_VERB_HI, "CGMS: iter %i rsq = %g rel = %g\n", iteration, rsqc, relnorm);
    if (iteration >= ia->restart || iteration >= ia->max_iter) break;
    if (rsqc * trueRsqFac < rsqstop) nextRsqCheck = iteration;
    if (relnorm * trueRelFac < relstop) nextRelCheck = iteration;
    if (nextRsqCheck <= iteration || (relstop > 0 && nextRelCheck <= iteration)) {
      if (yAy > 0) {
        dcx yAx = B::cdot(Ay, out[imin], q);
        B::caxpy(out[imin], dcx{-yAx.re / yAy, -yAx.im / yAy}, y, q);
      }
      double xAx = L.d2n(Mp, out[imin]);
      iteration++;
      if (xAx <= 0) break;
      dcx xr = B::cdot(out[imin], ry, q);
      B::caxpy(y, dcx{xr.re / xAx, xr.im / xAx}, out[imin], q);
      yAy = L.d2n(Ay, y);
      iteration++;
      B::axpby(ry, 1.0, in, -1.0, Ay, q);
      B::zero(out[imin], q);
    }
    if (nextRsqCheck <= iteration) {
      double tr2;
      if (irsq == imin) {
        tr2 = B::norm2(ry, q);
      } else {
        double xAx = L.d2n(Mp, out[irsq]);
        iteration++;
        if (xAx <= 0) break;
        B::axpy(Mp, -1.0, in, q);
        tr2 = B::norm2(Mp, q);
      }
      log0(QOP_VERB_MED, "CGMS: %i: rsq: %g  tr2: %g\n", iteration, rsq, tr2);
      if (tr2 <= rsqstop) { rsq = tr2; break; }
      if (tr2 > 2 * rsq) break;
      trueRsqFac = tr2 / rsq;
      nextRsqCheck += rsqCheckInterval;
    }
    if (relstop > 0 && nextRelCheck <= iteration) {
      double xAx = L.d2n(Mp, out[irel]);
      iteration++;
      if (xAx <= 0) break;
      B::axpy(Mp, -1.0, in, q);
      double rel2 = relnorm2<T>(Mp, out[irel], eo);
      if (rel2 <= relstop) { relnorm = rel2; break; }
      trueRelFac = rel2 / relnorm;
      nextRelCheck += relCheckInterval;
      relnorm = rel2;
    }
    a[imin] = rsq / oldrsq;
    B::xpay(p, r, a[imin], q);
    for (int i = 0; i < ns; i++) {
      if (i == imin) continue;
      double c2v = z[i] * b[imin];
      a[i] = (c2v != 0.0) ? a[imin] * zn[i] * b[i] / c2v : 0;
    }
    for (int i = 0; i < ns; i++)
      if (i != imin) B::axpby(pm[i], a[i], pm[i], zn[i], r, q);
    for (int i = 0; i < ns; i++) { bo[i] = b[i]; zo[i] = z[i]; z[i] = zn[i]; }
  }
  B::copy(out[imin], y, q);
  for (int i = 0; i < ns; i++) {
    double s = zn[i] * zn[i];
    ra[i]->final_rsq = s * trueRsqFac * rsq / insq;
    ra[i]->final_rel = s * trueRelFac * relnorm;
    ra[i]->final_iter = iteration;
    ra[i]->final_restart = 0;
  }
  log0(QOP_VERB_MED, "CGMS: done: iter: %i  rsq: %g  rsq/insq: %g\n", iteration, rsq, rsq / insq);
}

// ---------------------------------------------------------------- refine
// r[i] on the opposite parity holds A out[i]; on return r[i] on insub holds
// in + scale*(D_ab D_ba out - m^2 out) and r2[i] its norm
template <typename T>
static void refine(FlaT<T> *f, c2<T> **out, c2<T> **in, c2<T> **r, double *r2, const double *m2, dcx *scale, int no,
                   int ineo, c2<T> **x, c2<T> **Ax, int nx, const int *oi, const int *xi, int ni, c2<T> *tv) {
  typedef Blas<T> B;
  const Geom &g = ctx().g;
  const int opeo = opp(ineo);
  const Range is = vrange(g, ineo), os = vrange(g, opeo);
  c2<T> **Aout = r;
  for (int i = 0; i < nx; i++) Dslash<T>::apply(f, 0, Ax[i], x[i], opeo, ineo);
  std::vector<double> x2(nx + 1), Ax2(nx + 1);
  for (int i = 0; i < nx; i++) { x2[i] = B::norm2(x[i], is); Ax2[i] = B::norm2(Ax[i], os); }
  for (int i = 0; i < ni; i++) {
    int ko = oi[i], kx = nx > 0 ? xi[i] : 0;
    dcx z{0, 0}, Az{0, 0}, s{0, 0}, sx{0, 0};
    double d = 0;
    Dslash<T>::apply(f, 0, Aout[ko], out[ko], opeo, ineo);
    if (nx > 0) {
      z = B::cdot(x[kx], out[ko], is);
      Az = B::cdot(Ax[kx], Aout[ko], os);
      d = Ax2[kx] + m2[ko] * x2[kx];
    }
    if (d != 0) {
      double di = 1 / d, dim2 = di * m2[ko];
      s = dim2 * z + di * Az;
      B::caxpy(out[ko], dcx{-s.re, -s.im}, x[kx], is);
      B::caxpy(Aout[ko], dcx{-s.re, -s.im}, Ax[kx], os);
      z = B::cdot(x[kx], in[ko], is);
      sx = di * z;
    }
    z = B::cdot(out[ko], in[ko], is);
    double o2 = B::norm2(out[ko], is), Ao2 = B::norm2(Aout[ko], os);
    d = Ao2 + m2[kx] * o2;   // the reference indexes m2 by kx here
    if (d != 0) {
      double di = 1 / d;
      s = di * z;
      scale[ko] = s;
      if (nx > 0) {
        dcx zz = cdiv(sx, s);
        B::caxpy(out[ko], zz, x[kx], is);
        B::caxpy(Aout[ko], zz, Ax[kx], os);
      }
    } else {
      scale[ko] = sx;
      if (nx > 0) { B::copy(out[ko], x[kx], is); B::copy(Aout[ko], Ax[kx], os); }
    }
  }
  for (int i = 0; i < no; i++) {
    Dslash<T>::apply(f, 0, tv, Aout[i], ineo, opeo);
    B::axpy(tv, -m2[i], out[i], is);
    B::caxpby(r[i], scale[i], tv, in[i], is);
    r2[i] = B::norm2(r[i], is);
  }
}

template <typename T> static FlaT<float> *shadow32(FlaT<T> *f) {
  if constexpr (std::is_same<T, float>::value) {
    return f;
  } else {
    if (!f->shadow32) f->shadow32 = (void *)fla_convert<float, double>(f);
    return (FlaT<float> *)f->shadow32;
  }
}

// inner multi-shift solve of solve_multi: FP64 reference CGMS, the
// reference's single-precision restart (mixed_rsq), or the B200 reliable-
// update solver (prec_sloppy < 64)
template <typename T>
static void inner_cgms(FlaT<T> *f, LinOp<T> &L, QOP_invert_arg_t *ia, QOP_resid_arg_t **xra, const double *m2s, int nm,
                       c2<T> **x, c2<T> *rhs, c2<T> *cgp, int ineo, bool mixed) {
  const Geom &g = ctx().g;
  const int prec = sloppy_prec();
  if constexpr (std::is_same<T, double>::value) {
    if (prec < 64 && mixed_cgms(L, ia, xra, m2s, nm, x, rhs, ineo, prec)) return;
  }
  if (std::is_same<T, double>::value && mixed) {
    // asqtad_invert_p.c:510-537: single-precision links and vectors
    FlaT<float> *f32 = shadow32(f);
    const Range is = vrange(g, ineo);
    Tmp<float> rf, tf, pf;
    std::vector<std::unique_ptr<Tmp<float>>> xfo;
    std::vector<c2<float> *> xf(nm);
    for (int i = 0; i < nm; i++) { xfo.emplace_back(new Tmp<float>()); xf[i] = *xfo.back(); }
    convert<float, T>(rf, rhs, is);
    std::vector<double> m2f(nm);
    for (int i = 0; i < nm; i++) m2f[i] = (double)(float)m2s[i];
    LinOp<float> Lf{f32, (double)(float)L.mass, L.eo, tf};
    cgms<float>(Lf, ia, xra, m2f.data(), nm, xf.data(), rf, pf, ineo);
    for (int i = 0; i < nm; i++) convert<T, float>(x[i], xf[i], is);
    return;
  }
  cgms<T>(L, ia, xra, m2s, nm, x, rhs, cgp, ineo);
}

// ---------------------------------------------------------------- solve_multi
template <typename T>
void solve_multi(QOP_info_t *info, FlaT<T> *f, QOP_invert_arg_t *ia, QOP_resid_arg_t **ra, const double *masses,
                 c2<T> **out, c2<T> **in, int nsolve) {
  typedef Blas<T> B;
  const Geom &g = ctx().g;
  const int ineo = ia->evenodd;
  if (ineo == QOP_EVENODD) {
    for (int i = 0; i < nsolve; i++) invert<T>(info, f, ia, ra[i], masses[i], out[i], in[i]);
    return;
  }
  if constexpr (std::is_same<T, double>::value) {
    if (sloppy_prec() < 64 && nsolve > 1 && !ctx().dd) {   // batched solver: single block only
      solve_multi_mixed(info, f, ia, ra, masses, out, in, nsolve);
      return;
    }
  }
  const int opeo = opp(ineo);
  const Range is = vrange(g, ineo);
  double dtime = 0;
  std::vector<double> in2(nsolve), r2(nsolve), r2stop(nsolve), mass2(nsolve), m2s(nsolve);
  std::vector<dcx> scale(nsolve, dcx{0, 0});
  std::vector<int> oi(nsolve), xi(nsolve);
  int nm = 0, iter = 0, nrestart = -1;
  const int max_iter = ia->max_iter, max_restarts = ia->max_restarts;
  const double mixedrsq = ia->mixed_rsq;
  Tmp<T> tv, cgp, optmp;
  std::vector<std::unique_ptr<Tmp<T>>> rr(nsolve);
  std::vector<c2<T> *> r(nsolve);
  for (int i = 0; i < nsolve; i++) {
    in2[i] = B::norm2(in[i], is);
    need_finite(in2[i], "solve: source norm");
  }
  for (int i = 0; i < nsolve; i++) {
    r2stop[i] = ra[i]->rsqmin * in2[i];
    mass2[i] = masses[i] * masses[i];
    log0(QOP_VERB_MED, "SOLVE: %i mass: %g rsqmin: %g rsqstop: %g relmin: %g\n", i, masses[i], ra[i]->rsqmin,
         r2stop[i], ra[i]->relmin);
    oi[i] = i;
    int j = nm;
    while (j > 0 && mass2[i] < m2s[j - 1]) j--;
    if (j == nm || m2s[j] != mass2[i]) {
      for (int k = nm; k > j; k--) m2s[k] = m2s[k - 1];
      m2s[j] = mass2[i];
      nm++;
    }
    rr[i].reset(new Tmp<T>());
    r[i] = *rr[i];
    Dslash<T>::apply(f, 0, r[i], out[i], opeo, ineo);
  }
  for (int i = 0; i < nsolve; i++) {
    int j = 0;
    while (j < nm - 1 && m2s[j] != mass2[i]) j++;
    xi[i] = j;
  }
  QOP_resid_arg_t resarg0 = QOP_RESID_ARG_DEFAULT;
  resarg0.rsqmin = 0;
  resarg0.relmin = 0;
  std::vector<QOP_resid_arg_t *> xra(nm);
  std::vector<std::unique_ptr<Tmp<T>>> xx(nm);
  std::vector<c2<T> *> x(nm);
  const double m20 = m2s[0];
  LinOp<T> L{f, std::sqrt(m20), ineo, optmp};
  for (int i = 0; i < nm; i++) { m2s[i] -= m20; xx[i].reset(new Tmp<T>()); x[i] = *xx[i]; }
  refine<T>(f, out, in, r.data(), r2.data(), mass2.data(), scale.data(), nsolve, ineo, nullptr, nullptr, 0, oi.data(),
            nullptr, nsolve, tv);
  while (true) {
    for (int i = 0; i < nsolve; i++)
      ra[i]->final_rel = ra[i]->relmin > 0 ? relnorm2<T>(r[i], out[i], ineo) : 1;
    int imax = 0, usingrel = 0;
    double r2max = 0, r2stopmax = 1, in2max = 1, rsqminfac = 1;
    for (int i = 0; i < nsolve; i++) {
      double r2i = r2[i], r2stopi = r2stop[i], in2i = in2[i], rsqminfaci = 1;
      int usingreli = 0;
      if (ra[i]->final_rel * r2stopi < r2i * ra[i]->relmin) {
        r2i = ra[i]->final_rel; r2stopi = ra[i]->relmin; in2i = 1; rsqminfaci = 1e-10; usingreli = 1;
      }
      double aa = r2i * r2stopmax, bb = r2max * r2stopi;
      if (aa > bb * 1.01 || (aa * 1.01 >= bb && mass2[i] < mass2[imax])) {
        imax = i; r2max = r2i; r2stopmax = r2stopi; in2max = in2i; rsqminfac = rsqminfaci; usingrel = usingreli;
      }
      log0(QOP_VERB_MED, "SOLVE[%i]: rsq = %g rel = %g\n", i, r2[i] / in2[i], ra[i]->final_rel);
    }
    log0(QOP_VERB_LOW, "SOLVE: its: %i worst: %i mass: %g rsq: %g/%g rel: %g/%g\n", iter, imax, masses[imax],
         r2[imax] / in2[imax], ra[imax]->rsqmin, ra[imax]->final_rel, ra[imax]->relmin);
    if (r2max <= r2stopmax || nrestart >= max_restarts || iter >= max_iter) break;
    for (int i = 0; i < nm; i++) {
      xra[i] = (i == xi[imax]) ? ra[imax] : &resarg0;
      B::zero(x[i], vrange(g, QOP_EVENODD));
    }
    const double rsqminold = ra[imax]->rsqmin;
    ra[imax]->rsqmin = r2stopmax / r2max;
    if (ra[imax]->rsqmin >= 1) ra[imax]->rsqmin = in2max * r2stopmax / r2max;
    ra[imax]->rsqmin *= rsqminfac;
    ia->max_iter = max_iter - iter;
    bool mixed = false;
    if (std::is_same<T, double>::value) {
      mixed = r2max > mixedrsq * in2max;
      if (mixed && mixedrsq > rsqminold) ra[imax]->rsqmin = mixedrsq * in2max / r2max;
    }
    double t0 = wtime();
    inner_cgms<T>(f, L, ia, xra.data(), m2s.data(), nm, x.data(), r[imax], cgp, ineo, mixed);
    dtime += wtime() - t0;
    iter += ra[imax]->final_iter;
    nrestart++;
    ra[imax]->rsqmin = rsqminold;
    if (usingrel) {
      for (int i = 0; i < nsolve; i++) {
        int ko = oi[i], kx = xi[i];
        if (norm2(scale[ko]) == 0.0) B::copy(out[ko], x[kx], is);
        else B::caxpy(out[ko], cdiv(dcx{1, 0}, scale[ko]), x[kx], is);
      }
      refine<T>(f, out, in, r.data(), r2.data(), mass2.data(), scale.data(), nsolve, ineo, nullptr, nullptr, 0,
                oi.data(), nullptr, nsolve, tv);
    } else {
      refine<T>(f, out, in, r.data(), r2.data(), mass2.data(), scale.data(), nsolve, ineo, x.data(), x.data(), nm,
                oi.data(), xi.data(), nsolve, tv);
    }
  }
  ia->max_iter = max_iter;
  for (int i = 0; i < nsolve; i++) {
    B::cscale(tv, masses[i] * scale[i], out[i], is);
    B::copy(out[i], tv, is);
    ra[i]->final_iter = iter;
    ra[i]->final_rsq = in2[i] > 0 ? r2[i] / in2[i] : 0;
    ra[i]->final_restart = nrestart > 0 ? nrestart : 0;
  }
  const double nflop = 0.5 * (20 * 3 + 2 * 8 * 3 * 3 * f->nlinks), nflopm = 0.5 * 10 * 3;
  sync();
  if (info) {
    info->final_sec = dtime;
    info->final_flop = (nflop + nflopm * (nm - 1)) * iter * (double)g.V;
    info->status = QOP_SUCCESS;
  }
  log0(QOP_VERB_LOW, "SOLVE: its: %i  sec: %g\n", iter, dtime);
}

// ---------------------------------------------------------------- invert
template <typename T>
void invert(QOP_info_t *info, FlaT<T> *f, QOP_invert_arg_t *ia, QOP_resid_arg_t *ra, double mass, c2<T> *out,
            const c2<T> *in) {
  typedef Blas<T> B;
  if (ia->evenodd != QOP_EVENODD) {
    c2<T> *o[1] = {out}, *i_[1] = {(c2<T> *)in};
    QOP_resid_arg_t *rr[1] = {ra};
    double m[1] = {mass};
    solve_multi<T>(info, f, ia, rr, m, o, i_, 1);
    return;
  }
  const Geom &g = ctx().g;
  const double nflop = 0.5 * (20 * 3 + 2 * 8 * 3 * 3 * f->nlinks);
  double dtime = 0;
  int iter = 0;
  const int max_iter_old = ia->max_iter, max_restarts_old = ia->max_restarts;
  int nrestart = -1, max_restarts = ia->max_restarts;
  if (max_restarts <= 0) max_restarts = 5;
  const int ineo = ia->evenodd;
  const Range is = vrange(g, ineo);
  double insqe = 0, insqo = 0;
  if (ineo != QOP_ODD) insqe = B::norm2(in, vrange(g, QOP_EVEN));
  if (ineo != QOP_EVEN) insqo = B::norm2(in, vrange(g, QOP_ODD));
  const double insq = insqe + insqo;
  need_finite(insq, "invert: source norm");
  const int cgeo = insqe >= insqo ? QOP_EVEN : QOP_ODD;
  const Range cs = vrange(g, cgeo), ocs = vrange(g, opp(cgeo));
  Tmp<T> cgp, cgr, tmp2, qin, qout, optmp;
  LinOp<T> L{f, mass, cgeo, optmp};
  B::copy(tmp2, in, is);
  Dslash<T>::apply(f, mass, qin, tmp2, cgeo, opp(cgeo));          // project (:80-89)
  B::axpby(qin, mass, tmp2, -1.0, qin, cs);
  if (ineo == cgeo) B::zero(qin, ocs); else B::copy(qin, in, ocs);
  const double pinsq = B::norm2(qin, cs);
  const double rsqfac = mass * mass * insq / pinsq;
  B::copy(qout, out, cs);
  const double rsqstop = insq * ra->rsqmin;
  log0(QOP_VERB_LOW, "ASQTAD_INVERT: rsqstop = %g\n", rsqstop);
  double rsq = 0, relnorm = 1.;
  const double rsqminold = ra->rsqmin, relminold = ra->relmin;
  ra->rsqmin = 0.99 * rsqminold * rsqfac;
  ra->relmin = 0.99 * relminold;
  ia->max_restarts = 0;
  do {
    double t0 = wtime();
    if (ctx().opt.cgtype == 1) eigcg<T>(L, ia, ra, qout, qin, cgp, cgeo, f);   // asqtad_invert_p.c:767-770
    else cg<T>(L, ia, ra, qout, qin, cgp, cgeo);
    dtime += wtime() - t0;
    iter += ra->final_iter;
    B::copy(cgr, qout, cs);                                      // reconstruct (:92-100)
    Dslash<T>::apply(f, mass, qout, cgr, opp(cgeo), cgeo);
    B::axpby(qout, 1.0 / mass, qin, -1.0 / mass, qout, ocs);
    Dslash<T>::apply(f, mass, cgr, qout, ineo, QOP_EVENODD);
    B::axpy(cgr, -1.0, in, is);
    rsq = B::norm2(cgr, is);
    ra->rsqmin *= 0.99;
    if (ra->relmin > 0) {
      relnorm = relnorm2<T>(cgr, qout, ineo);
      ra->relmin = 0.99 * ra->final_rel / relnorm * relminold;
    }
    log0(QOP_VERB_LOW, "ASQTAD_INVERT: iter %i rsq = %g rel = %g\n", iter, rsq, relnorm);
    ia->max_iter = max_iter_old - iter;
  } while ((++nrestart < max_restarts) && (ia->max_iter > 0) && (rsq > rsqstop) && (relnorm > ra->relmin));
  B::copy(out, qout, is);
  ia->max_iter = max_iter_old;
  ia->max_restarts = max_restarts_old;
  ra->rsqmin = rsqminold;
  ra->relmin = relminold;
  ra->final_iter = iter;
  ra->final_rsq = insq == 0. ? 0 : rsq / insq;
  ra->final_rel = relnorm;
  ra->final_restart = nrestart;
  sync();
  if (info) {
    info->final_sec = dtime;
    info->final_flop = nflop * ra->final_iter * (double)g.V;
    info->status = QOP_SUCCESS;
  }
}

// ---------------------------------------------------------------- invert_multi
template <typename T>
void invert_multi(QOP_info_t *info, FlaT<T> *f, QOP_invert_arg_t *ia, QOP_resid_arg_t **ra[], double *masses[],
                  int nmass[], c2<T> **out[], c2<T> *in[], int nsrc) {
  typedef Blas<T> B;
  const Geom &g = ctx().g;
  if (ia->evenodd != QOP_EVENODD) {
    int nsolve = 0;
    for (int i = 0; i < nsrc; i++) nsolve += nmass[i];
    std::vector<QOP_resid_arg_t *> rr;
    std::vector<double> ms;
    std::vector<c2<T> *> o, in_;
    for (int i = 0; i < nsrc; i++)
      for (int j = 0; j < nmass[i]; j++) {
        rr.push_back(ra[i][j]); ms.push_back(masses[i][j]); o.push_back(out[i][j]); in_.push_back(in[i]);
      }
    solve_multi<T>(info, f, ia, rr.data(), ms.data(), o.data(), in_.data(), nsolve);
    return;
  }
  const double nflop = 0.5 * (20 * 3 + 2 * 8 * 3 * 3 * f->nlinks), nflopm = 0.5 * 10 * 3;
  double flop = 0, t0 = wtime();
  const int cgeo = QOP_EVEN;
  log0(QOP_VERB_LOW, "warning: QOP_asqtad_invert_multi on ALL subset not supported yet!\n");
  const Range cs = vrange(g, cgeo);
  Tmp<T> cgp, optmp;
  if (nsrc == 2 && nmass[0] == 1 && nmass[1] == 1 && masses[0][0] != masses[1][0]) {
    double shifts[2], rsqsave[2];
    int imin = 0;
    c2<T> *incv[2], *outcv[2];
    QOP_resid_arg_t *rr[2];
    for (int i = 0; i < 2; i++) {
      shifts[i] = masses[i][0] * masses[i][0];
      if (shifts[i] < shifts[imin]) imin = i;
      incv[i] = in[i]; outcv[i] = out[i][0]; rr[i] = ra[i][0];
    }
    const double gm = masses[imin][0];
    for (int i = 0; i < 2; i++) shifts[i] -= gm * gm;
    const double st = 1 / (shifts[1] - shifts[0]);
    Tmp<T> x0, src;
    B::axpby(x0, st, incv[1], -st, incv[0], cs);
    B::copy(cgp, x0, cs);
    LinOp<T> L{f, gm, cgeo, optmp};
    L.d2(src, cgp);
    B::axpby(src, 1.0, incv[imin], -1.0, src, cs);
    const double rsq1 = B::norm2(src, cs);
    for (int i = 0; i < 2; i++) {
      double rsq0 = B::norm2(incv[i], cs);
      rsqsave[i] = ra[i][0]->rsqmin;
      ra[i][0]->rsqmin *= rsq0 / rsq1;
    }
    cgms<T>(L, ia, rr, shifts, 2, outcv, src, cgp, cgeo);
    flop += (nflop + nflopm) * rr[imin]->final_iter * (double)g.V;
    for (int i = 0; i < 2; i++) {
      ra[i][0]->rsqmin = rsqsave[i];
      B::axpy(outcv[i], 1.0, x0, cs);
    }
  } else {
    for (int i = 0; i < nsrc; i++) {
      std::vector<double> shifts(nmass[i]);
      int jmin = 0;
      for (int j = 0; j < nmass[i]; j++) {
        shifts[j] = masses[i][j] * masses[i][j];
        if (shifts[j] < shifts[jmin]) jmin = j;
      }
      const double gm = masses[i][jmin];
      for (int j = 0; j < nmass[i]; j++) shifts[j] -= gm * gm;
      LinOp<T> L{f, gm, cgeo, optmp};
      cgms<T>(L, ia, ra[i], shifts.data(), nmass[i], out[i], in[i], cgp, cgeo);
      flop += (nflop + nflopm * (nmass[i] - 1)) * ra[i][0]->final_iter * (double)g.V;
    }
  }
  for (int i = 0; i < nsrc; i++)
    for (int j = 0; j < nmass[i]; j++) B::scale(out[i][j], masses[i][j], out[i][j], cs);
  sync();
  if (info) {
    info->final_sec = wtime() - t0;
    info->final_flop = flop;
    info->status = QOP_SUCCESS;
  }
}

#define INST(T)                                                                                                  \
  template void cg<T>(LinOp<T> &, QOP_invert_arg_t *, QOP_resid_arg_t *, c2<T> *, const c2<T> *, c2<T> *, int);   \
  template void cgms<T>(LinOp<T> &, QOP_invert_arg_t *, QOP_resid_arg_t **, const double *, int, c2<T> **,        \
                        const c2<T> *, c2<T> *, int);                                                            \
  template void invert<T>(QOP_info_t *, FlaT<T> *, QOP_invert_arg_t *, QOP_resid_arg_t *, double, c2<T> *,       \
                          const c2<T> *);                                                                        \
  template void solve_multi<T>(QOP_info_t *, FlaT<T> *, QOP_invert_arg_t *, QOP_resid_arg_t **, const double *,  \
                               c2<T> **, c2<T> **, int);                                                         \
  template void invert_multi<T>(QOP_info_t *, FlaT<T> *, QOP_invert_arg_t *, QOP_resid_arg_t **[], double *[],   \
                                int[], c2<T> **[], c2<T> *[], int);
INST(float)
INST(double)

}  // namespace qopb
