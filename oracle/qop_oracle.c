/*
 * qop_oracle.c -- TEST INFRASTRUCTURE ONLY (see qop_oracle.h).
 *
 * FP64 CPU restatement of QOPQDP's asqtad/HISQ hot path.  Each routine
 * names the reference file:line whose algorithm it restates.  The
 * reference's QDP field operations become plain site loops over host
 * arrays; its QLA site algebra becomes the small complex helpers below.
 * Parity: pinned to the reference itself.  oracle/ref compiles the
 * reference's own asqtad/HISQ sources, unmodified, against a CPU stand-in
 * for the QDP/QLA/QMP calls they make (oracle/_ref/libqopref.so);
 * tests/test_ref_pin.py compares this file with that library (rephase,
 * asqtad and HISQ links, the nine Dslash cases, invert, invert_multi) and
 * with its committed outputs (tests/golden/qopref_4x4x4x4.npz); the
 * reference's check_op / check_resids identities (examples/asqtad_test.c:
 * 37-130) are checked too.
 */
#include "qop_oracle.h"
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex dc;
enum { EVEN = 0, ODD = 1, EVENODD = 2 };

struct or_lat {
  int L[4];
  long V, Vh;
  int *x;     /* V x 4 coordinates, by raw index            */
  long *nb;   /* V x 4 dirs x {+1,+3,-1,-3}: raw neighbours  */
};

struct or_fla {
  or_lat *g;
  int nlinks;       /* 16 with Naik, 8 without                          */
  dc *fwd[8];       /* fwd[2mu]=fat_mu/2, fwd[2mu+1]=long_mu/2 (or fat) */
  dc *bck[8];       /* bck[i](x) = -fwd[i](x - shift_i)^dagger          */
  dc *dbl[16];
  int dbl_mu[16], dbl_disp[16];
};

/* ------------------------------------------------------------------ */
/* threads                                                             */
/* ------------------------------------------------------------------ */
void or_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
int or_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* geometry: lib/layout_user.c:237-258 (index), :260-312 (coords)      */
/* lex index has x[0] slowest, x[3] fastest; even sites come first.    */
/* ------------------------------------------------------------------ */
static long lex_of(const int L[4], const int x[4]) {
  long l = 0;
  for (int i = 0; i < 4; i++) l = l * L[i] + x[i];
  return l;
}

long or_raw_index(const or_lat *g, const int x[4]) {
  long l = lex_of(g->L, x);
  int s = x[0] + x[1] + x[2] + x[3];
  return (s % 2 == 0) ? l / 2 : (l + g->V) / 2;
}

or_lat *or_lat_create(const int L[4]) {
  or_lat *g = calloc(1, sizeof(*g));
  g->V = 1;
  for (int i = 0; i < 4; i++) { g->L[i] = L[i]; g->V *= L[i]; }
  g->Vh = g->V / 2;
  g->x = malloc(sizeof(int) * 4 * g->V);
  g->nb = malloc(sizeof(long) * 16 * g->V);
#pragma omp parallel for
  for (long l = 0; l < g->V; l++) {
    int x[4];
    long t = l;
    for (int i = 3; i >= 0; i--) { x[i] = (int)(t % L[i]); t /= L[i]; }
    long idx = or_raw_index(g, x);
    memcpy(g->x + 4 * idx, x, sizeof(x));
  }
#pragma omp parallel for
  for (long idx = 0; idx < g->V; idx++) {
    const int *x = g->x + 4 * idx;
    static const int disp[4] = {1, 3, -1, -3};
    for (int mu = 0; mu < 4; mu++)
      for (int k = 0; k < 4; k++) {
        int y[4] = {x[0], x[1], x[2], x[3]};
        y[mu] = ((y[mu] + disp[k]) % g->L[mu] + g->L[mu]) % g->L[mu];
        g->nb[16 * idx + 4 * mu + k] = or_raw_index(g, y);
      }
  }
  return g;
}

void or_lat_destroy(or_lat *g) {
  if (!g) return;
  free(g->x); free(g->nb); free(g);
}
long or_lat_volume(const or_lat *g) { return g->V; }
void or_raw_coords(const or_lat *g, long idx, int x[4]) { memcpy(x, g->x + 4 * idx, 4 * sizeof(int)); }

long or_neighbor(const or_lat *g, long idx, int mu, int disp) {
  int y[4];
  or_raw_coords(g, idx, y);
  y[mu] = ((y[mu] + disp) % g->L[mu] + g->L[mu]) % g->L[mu];
  return or_raw_index(g, y);
}

static inline long nbr(const or_lat *g, long idx, int mu, int disp) {
  int k = disp == 1 ? 0 : disp == 3 ? 1 : disp == -1 ? 2 : disp == -3 ? 3 : -1;
  if (k < 0) return or_neighbor(g, idx, mu, disp);
  return g->nb[16 * idx + 4 * mu + k];
}

/* subsets: raw index ranges (qop_internal.h:64-65 qdpsub) */
static void sub_range(const or_lat *g, int eo, long *lo, long *hi) {
  if (eo == EVEN) { *lo = 0; *hi = g->Vh; }
  else if (eo == ODD) { *lo = g->Vh; *hi = g->V; }
  else { *lo = 0; *hi = g->V; }
}
static int opp(int eo) { return eo == EVEN ? ODD : eo == ODD ? EVEN : EVENODD; }

/* ------------------------------------------------------------------ */
/* 3x3 complex site algebra (QLA restated)                             */
/* ------------------------------------------------------------------ */
static inline void m_mul(dc *r, const dc *a, const dc *b) {        /* r = a b    */
  dc t[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      dc s = 0;
      for (int k = 0; k < 3; k++) s += a[3 * i + k] * b[3 * k + j];
      t[3 * i + j] = s;
    }
  memcpy(r, t, sizeof(t));
}
static inline void m_mul_na(dc *r, const dc *a, const dc *b) {     /* r = a b^+  */
  dc t[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      dc s = 0;
      for (int k = 0; k < 3; k++) s += a[3 * i + k] * conj(b[3 * j + k]);
      t[3 * i + j] = s;
    }
  memcpy(r, t, sizeof(t));
}
static inline void m_mul_an(dc *r, const dc *a, const dc *b) {     /* r = a^+ b  */
  dc t[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      dc s = 0;
      for (int k = 0; k < 3; k++) s += conj(a[3 * k + i]) * b[3 * k + j];
      t[3 * i + j] = s;
    }
  memcpy(r, t, sizeof(t));
}
static inline void mv_mul_acc(dc *r, const dc *m, const dc *v) {   /* r += m v   */
  for (int i = 0; i < 3; i++) {
    dc s = 0;
    for (int k = 0; k < 3; k++) s += m[3 * i + k] * v[k];
    r[i] += s;
  }
}
static inline void mav_mul(dc *r, const dc *m, const dc *v) {      /* r = m^+ v  */
  for (int i = 0; i < 3; i++) {
    dc s = 0;
    for (int k = 0; k < 3; k++) s += conj(m[3 * k + i]) * v[k];
    r[i] = s;
  }
}

/* ------------------------------------------------------------------ */
/* rephase: lib/common_p.c:455-526 (gauge field)                        */
/* ------------------------------------------------------------------ */
void or_rephase_G(const or_lat *g, double *links[4], const int r0[4],
                  const double *bc_reim, const int *signmask) {
  for (int i = 0; i < 4; i++) {
    int bc_dir = -1;
    dc ph = 1;
    if (bc_reim && (bc_reim[2 * i] != 1. || bc_reim[2 * i + 1] != 0.)) {
      bc_dir = i;
      ph = bc_reim[2 * i] + I * bc_reim[2 * i + 1];
    }
    int bits = signmask ? signmask[i] : 0;
    dc *m = (dc *)links[i];
    int n = g->L[i], org = r0 ? r0[i] : 0;
#pragma omp parallel for
    for (long s = 0; s < g->V; s++) {
      const int *x = g->x + 4 * s;
      dc f = 1;
      if (bc_dir >= 0) {
        int rshift = (x[bc_dir] + n - org) % n;
        if (rshift == n - 1) f *= ph;
      }
      if (bits) {
        int t = 0;
        for (int j = 0; j < 4; j++) t += ((bits >> j) & 1) * x[j];
        if (t & 1) f = -f;
      }
      if (f != 1) for (int e = 0; e < 9; e++) m[9 * s + e] *= f;
    }
  }
}

/* ------------------------------------------------------------------ */
/* smearing: lib/asqtad_dslash_p.c:391-455 (compute_gen_staple) and     */
/* :458-633 (make_imp_links, non-QLL branch)                            */
/* ------------------------------------------------------------------ */
/* staple of `link` in plane (mu,nu):
   upper(x) = U_nu(x) [link(x+nu) U_nu(x+mu)^+]
   lower(x) = [U_nu(y)^+ link(y)] U_nu(y+mu),  y = x - nu
   save != NULL: save = upper + lower, fl += coef*save
   save == NULL: fl += coef*upper; fl += coef*lower                    */
static void gen_staple(const or_lat *g, dc *save, int mu, int nu, const dc *link,
                       double coef, dc **gauge, dc *fl) {
#pragma omp parallel for
  for (long s = 0; s < g->V; s++) {
    dc t1[9], up[9], lo[9];
    long xpn = nbr(g, s, nu, 1), xpm = nbr(g, s, mu, 1);
    long y = nbr(g, s, nu, -1), ypm = nbr(g, y, mu, 1);
    m_mul_na(t1, link + 9 * xpn, gauge[nu] + 9 * xpm);
    m_mul(up, gauge[nu] + 9 * s, t1);
    m_mul_an(t1, gauge[nu] + 9 * y, link + 9 * y);
    m_mul(lo, t1, gauge[nu] + 9 * ypm);
    if (save) {
      for (int e = 0; e < 9; e++) {
        save[9 * s + e] = up[e] + lo[e];
        fl[9 * s + e] += coef * save[9 * s + e];
      }
    } else {
      for (int e = 0; e < 9; e++) fl[9 * s + e] += coef * up[e];
      for (int e = 0; e < 9; e++) fl[9 * s + e] += coef * lo[e];
    }
  }
}

void or_make_imp_links(const or_lat *g, const double coef[6], double *gfr[4],
                       double *gfLongr[4], double *flr[4], double *llr[4]) {
  dc *gf[4], *gfLong[4], *fl[4];
  for (int i = 0; i < 4; i++) {
    gf[i] = (dc *)gfr[i]; gfLong[i] = (dc *)gfLongr[i]; fl[i] = (dc *)flr[i];
  }
  double c1 = coef[0], c3 = coef[1], c5 = coef[2], c7 = coef[3], cL = coef[4];
  c1 -= 6 * cL;                           /* Lepage trick :531 */
  int have5 = c5 != 0 || c7 != 0 || cL != 0;
  int have3 = c3 != 0 || have5;
  size_t fsz = sizeof(dc) * 9 * g->V;
  dc *staple = malloc(fsz), *tmp1 = malloc(fsz);
  for (int dir = 0; dir < 4; dir++) {
#pragma omp parallel for
    for (long s = 0; s < 9 * g->V; s++) fl[dir][s] = c1 * gf[dir][s];
    if (!have3) continue;
    for (int nu = 0; nu < 4; nu++) {
      if (nu == dir) continue;
      gen_staple(g, staple, dir, nu, gf[dir], c3, gf, fl[dir]);
      if (cL != 0) gen_staple(g, NULL, dir, nu, staple, cL, gf, fl[dir]);
      if (c5 != 0 || c7 != 0) {
        for (int rho = 0; rho < 4; rho++) {
          if (rho == dir || rho == nu) continue;
          gen_staple(g, tmp1, dir, rho, staple, c5, gf, fl[dir]);
          if (c7 != 0)
            for (int sig = 0; sig < 4; sig++)
              if (sig != dir && sig != nu && sig != rho)
                gen_staple(g, NULL, dir, sig, tmp1, c7, gf, fl[dir]);
        }
      }
    }
  }
  if (llr) {                              /* Naik links :594-604 */
    double naik = coef[5];
    for (int dir = 0; dir < 4; dir++) {
      dc *ll = (dc *)llr[dir];
#pragma omp parallel for
      for (long s = 0; s < g->V; s++) {
        dc t[9];
        long x1 = nbr(g, s, dir, 1), x2 = nbr(g, x1, dir, 1);
        m_mul(t, gfLong[dir] + 9 * x1, gfLong[dir] + 9 * x2);
        m_mul(ll + 9 * s, gfLong[dir] + 9 * s, t);
        for (int e = 0; e < 9; e++) ll[9 * s + e] *= naik;
      }
    }
  }
  free(staple); free(tmp1);
}

/* ------------------------------------------------------------------ */
/* U(3) projection: lib/hisq_reunit_utilities_p.c:99-297                 */
/* W = V (V^+V)^{-1/2}: eigenvalues of Q=V^+V from the trigonometric     */
/* cubic solution, Q^{-1/2} = f0 + f1 Q + f2 Q^2.  The reference's SVD   */
/* fallback (:709+) is replaced by a Jacobi eigen-decomposition of Q:    */
/* for non-singular V both give the unique polar factor.                 */
/* ------------------------------------------------------------------ */
static dc det3(const dc *u) {
  dc m0 = u[4] * u[8] - u[5] * u[7];
  dc m1 = u[3] * u[8] - u[5] * u[6];
  dc m2 = u[3] * u[7] - u[4] * u[6];
  return u[0] * m0 - u[1] * m1 + u[2] * m2;
}

/* Hermitian 3x3 Jacobi: Q = Z diag(w) Z^+ */
static void herm_eig3(const dc *Qin, double w[3], dc Z[9]) {
  dc A[9];
  memcpy(A, Qin, sizeof(A));
  for (int i = 0; i < 9; i++) Z[i] = (i % 4 == 0) ? 1 : 0;
  for (int sweep = 0; sweep < 60; sweep++) {
    double off = 0;
    for (int p = 0; p < 3; p++)
      for (int q = p + 1; q < 3; q++) off += cabs(A[3 * p + q]) * cabs(A[3 * p + q]);
    if (off < 1e-34) break;
    for (int p = 0; p < 3; p++)
      for (int q = p + 1; q < 3; q++) {
        dc apq = A[3 * p + q];
        double r = cabs(apq);
        if (r < 1e-300) continue;
        double app = creal(A[4 * p]), aqq = creal(A[4 * q]);
        dc ph = apq / r;
        double theta = 0.5 * atan2(2 * r, aqq - app);
        double c = cos(theta), s = sin(theta);
        /* rotation G: columns p,q  ->  [c, s*conj(ph)... ] */
        dc gpp = c, gpq = s * ph, gqp = -s * conj(ph), gqq = c;
        /* A <- G^+ A G ; Z <- Z G, with G acting on columns p,q */
        for (int k = 0; k < 3; k++) {              /* A G */
          dc akp = A[3 * k + p], akq = A[3 * k + q];
          A[3 * k + p] = akp * gpp + akq * gqp;
          A[3 * k + q] = akp * gpq + akq * gqq;
          dc zkp = Z[3 * k + p], zkq = Z[3 * k + q];
          Z[3 * k + p] = zkp * gpp + zkq * gqp;
          Z[3 * k + q] = zkp * gpq + zkq * gqq;
        }
        for (int k = 0; k < 3; k++) {              /* G^+ (A G) */
          dc apk = A[3 * p + k], aqk = A[3 * q + k];
          A[3 * p + k] = conj(gpp) * apk + conj(gqp) * aqk;
          A[3 * q + k] = conj(gpq) * apk + conj(gqq) * aqk;
        }
      }
  }
  for (int i = 0; i < 3; i++) w[i] = creal(A[4 * i]);
}

int or_u3_un_analytic(const double Vr[18], double Wr[18], int allow_svd,
                      double svd_rel_err, double svd_abs_err) {
  const dc *V = (const dc *)Vr;
  dc *W = (dc *)Wr;
  const double EPS = 1.0e-14, PI = 3.14159265358979323846;
  double det_check = 0;
  if (allow_svd) {
    dc d = det3(V);
    det_check = creal(d) * creal(d) + cimag(d) * cimag(d);
  }
  dc Q[9], Q2[9], Q3[9];
  m_mul_an(Q, V, V);
  m_mul(Q2, Q, Q);
  m_mul(Q3, Q2, Q);
  double c0 = creal(Q[0] + Q[4] + Q[8]);
  double c1 = creal(Q2[0] + Q2[4] + Q2[8]) / 2;
  double c2 = creal(Q3[0] + Q3[4] + Q3[8]) / 3;
  double S = c1 / 3 - c0 * (c0 / 18), g0, g1, g2;
  if (fabs(S) < EPS) {
    g0 = g1 = g2 = c0 / 3;
  } else {
    double R = c2 / 2 - c0 * (c1 / 3) + c0 * c0 * (c0 / 27);
    S = sqrt(S);
    double RoS = R / (S * S * S), theta;
    if (!(fabs(RoS) < 1.0)) theta = R > 0 ? 0.0 : PI;
    else theta = acos(RoS);
    double th3 = theta / 3, pi23 = (2 * PI) / 3;
    g0 = c0 / 3 + 2 * S * cos(th3);
    g1 = c0 / 3 + 2 * S * cos(th3 + pi23);
    g2 = c0 / 3 + 2 * S * cos(th3 + 2 * pi23);
  }
  int svd = 0;
  if (allow_svd) {
    if (det_check != 0 && fabs(det_check - g0 * g1 * g2) / fabs(det_check) > svd_rel_err) svd = 1;
    if (det_check < svd_abs_err) svd = 1;
  }
  if (svd) {
    double w[3]; dc Z[9], S2[9];
    herm_eig3(Q, w, Z);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        dc s = 0;
        for (int k = 0; k < 3; k++) s += Z[3 * i + k] * (w[k] > 0 ? 1.0 / sqrt(w[k]) : 0.0) * conj(Z[3 * j + k]);
        S2[3 * i + j] = s;
      }
    m_mul(W, V, S2);
    return 1;
  }
  double g0sq = sqrt(g0), g1sq = sqrt(g1), g2sq = sqrt(g2);
  double us = g1sq + g2sq, ws = g1sq * g2sq, vs = g0sq * us + ws;
  us += g0sq;
  ws *= g0sq;
  double denom = ws * (us * vs - ws);
  double f0 = (us * vs * vs - ws * (us * us + vs)) / denom;
  double f1 = (2 * us * vs - ws - us * us * us) / denom;
  double f2 = us / denom;
  dc S2[9];
  for (int e = 0; e < 9; e++) S2[e] = f1 * Q[e] + f2 * Q2[e];
  S2[0] += f0; S2[4] += f0; S2[8] += f0;
  m_mul(W, V, S2);
  return 0;
}

int or_u3reunit(const or_lat *g, double *Vf, double *Wf) {
  int nsvd = 0;
#pragma omp parallel for reduction(+:nsvd)
  for (long s = 0; s < g->V; s++)
    nsvd += or_u3_un_analytic(Vf + 18 * s, Wf + 18 * s, 1, 1e-8, 1e-8);
  return nsvd;
}

/* HISQ: lib/hisq_links_p.c:62-256 (n_naiks = 1 path; difference links only
   when n_naiks > 1, which the oracle does not need) */
int or_hisq_links(const or_lat *g, const double h[18], double *gauge[4],
                  double *fat[4], double *lng[4], double *Wout[4]) {
  size_t fsz = sizeof(double) * 18 * g->V;
  double *Vl[4], *Wl[4];
  for (int i = 0; i < 4; i++) { Vl[i] = malloc(fsz); Wl[i] = Wout ? Wout[i] : malloc(fsz); }
  double c7[6] = {h[0], h[1], h[2], h[3], h[13] != 0 ? h[4] : 0.0, 0.0};
  /* fat7 stage: create_L_from_G scales by 1/2, the caller scales back by 2,
     so the fat7 links are make_imp_links' output as is */
  or_make_imp_links(g, c7, gauge, gauge, Vl, NULL);
  int nsvd = 0;
  for (int i = 0; i < 4; i++) {
#pragma omp parallel for reduction(+:nsvd)
    for (long s = 0; s < g->V; s++)
      nsvd += or_u3_un_analytic(Vl[i] + 18 * s, Wl[i] + 18 * s, h[14] != 0, h[15], h[16]);
  }
  double ca[6] = {h[5], h[6], h[7], h[8], h[9], h[10]};
  or_make_imp_links(g, ca, Wl, Wl, fat, ca[5] != 0 ? lng : NULL);
  for (int i = 0; i < 4; i++) { free(Vl[i]); if (!Wout) free(Wl[i]); }
  return nsvd;
}

/* ------------------------------------------------------------------ */
/* link object: lib/asqtad_dslash_p.c:152-223 (convert_L: scale by 1/2) */
/* and :79-133 (double_store: bck(x) = -fwd(x - shift)^+)               */
/* ------------------------------------------------------------------ */
or_fla *or_fla_create(or_lat *g, double *fat[4], double *lng[4]) {
  or_fla *f = calloc(1, sizeof(*f));
  f->g = g;
  f->nlinks = lng ? 16 : 8;
  int nl2 = f->nlinks / 2;
  size_t fsz = sizeof(dc) * 9 * g->V;
  for (int i = 0; i < nl2; i++) {
    f->fwd[i] = malloc(fsz);
    f->bck[i] = malloc(fsz);
    const double *src = lng ? (i % 2 ? lng[i / 2] : fat[i / 2]) : fat[i];
#pragma omp parallel for
    for (long s = 0; s < 9 * g->V; s++)
      f->fwd[i][s] = 0.5 * (src[2 * s] + I * src[2 * s + 1]);
  }
  for (int i = 0; i < nl2; i++) {
    int mu = lng ? i / 2 : i, d = (lng && (i % 2)) ? 3 : 1;
#pragma omp parallel for
    for (long s = 0; s < g->V; s++) {
      long y = nbr(g, s, mu, -d);
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
          f->bck[i][9 * s + 3 * a + b] = -conj(f->fwd[i][9 * y + 3 * b + a]);
    }
  }
  if (lng) {
    for (int mu = 0; mu < 4; mu++) {
      f->dbl[4 * mu] = f->fwd[2 * mu];     f->dbl_mu[4 * mu] = mu;     f->dbl_disp[4 * mu] = 1;
      f->dbl[4 * mu + 1] = f->fwd[2 * mu + 1]; f->dbl_mu[4 * mu + 1] = mu; f->dbl_disp[4 * mu + 1] = 3;
      f->dbl[4 * mu + 2] = f->bck[2 * mu];     f->dbl_mu[4 * mu + 2] = mu; f->dbl_disp[4 * mu + 2] = -1;
      f->dbl[4 * mu + 3] = f->bck[2 * mu + 1]; f->dbl_mu[4 * mu + 3] = mu; f->dbl_disp[4 * mu + 3] = -3;
    }
  } else {
    for (int mu = 0; mu < 4; mu++) {
      f->dbl[2 * mu] = f->fwd[mu];     f->dbl_mu[2 * mu] = mu;     f->dbl_disp[2 * mu] = 1;
      f->dbl[2 * mu + 1] = f->bck[mu]; f->dbl_mu[2 * mu + 1] = mu; f->dbl_disp[2 * mu + 1] = -1;
    }
  }
  return f;
}

void or_fla_destroy(or_fla *f) {
  if (!f) return;
  for (int i = 0; i < f->nlinks / 2; i++) { free(f->fwd[i]); free(f->bck[i]); }
  free(f);
}

/* ------------------------------------------------------------------ */
/* vector BLAS over a raw-index range (QDP_V_* restated)               */
/* ------------------------------------------------------------------ */
typedef struct { long lo, hi; } rng;
static rng R(const or_lat *g, int eo) { rng r; sub_range(g, eo, &r.lo, &r.hi); return r; }
#define VLOOP(r) _Pragma("omp parallel for") for (long e = 3 * (r).lo; e < 3 * (r).hi; e++)

static double v_norm2(const dc *a, rng r) {
  double s = 0;
#pragma omp parallel for reduction(+:s)
  for (long e = 3 * r.lo; e < 3 * r.hi; e++) s += creal(a[e]) * creal(a[e]) + cimag(a[e]) * cimag(a[e]);
  return s;
}
static dc v_dot(const dc *a, const dc *b, rng r) {    /* sum conj(a) b */
  double sr = 0, si = 0;
#pragma omp parallel for reduction(+:sr,si)
  for (long e = 3 * r.lo; e < 3 * r.hi; e++) {
    dc t = conj(a[e]) * b[e];
    sr += creal(t); si += cimag(t);
  }
  return sr + I * si;
}
static double v_redot(const dc *a, const dc *b, rng r) { return creal(v_dot(a, b, r)); }
static void v_zero(dc *a, rng r) { VLOOP(r) a[e] = 0; }
static void v_copy(dc *d, const dc *s, rng r) { if (d != s) { VLOOP(r) d[e] = s[e]; } }
static dc *v_new(const or_lat *g) { return calloc(3 * g->V, sizeof(dc)); }

double or_relnorm2(const or_lat *g, const double *rr, const double *xx, int eo) {
  /* lib/invert_utilities_p.c:1-40 */
  const dc *r = (const dc *)rr, *x = (const dc *)xx;
  rng q = R(g, eo);
  double s = 0;
#pragma omp parallel for reduction(+:s)
  for (long i = q.lo; i < q.hi; i++) {
    double xn = 0, rn = 0;
    for (int c = 0; c < 3; c++) {
      xn += creal(x[3 * i + c]) * creal(x[3 * i + c]) + cimag(x[3 * i + c]) * cimag(x[3 * i + c]);
      rn += creal(r[3 * i + c]) * creal(r[3 * i + c]) + cimag(r[3 * i + c]) * cimag(r[3 * i + c]);
    }
    s += (xn == 0.) ? 1. : rn / xn;
  }
  return s / (double)(q.hi - q.lo);
}

/* ------------------------------------------------------------------ */
/* Dslash: lib/asqtad_dslash_p.c:1048-1092 (dispatch), :1246-1279 (hop, */
/* style 1: dest = sum_i dbllinks[i](x) src(x + shift_i))               */
/* ------------------------------------------------------------------ */
static void hop(or_fla *f, dc *dest, const dc *src, int eo) {
  const or_lat *g = f->g;
  rng r = R(g, eo);
  const dc *s = src;
  dc *tmp = NULL;
  if (dest == src) {               /* the reference hops from a temp copy */
    tmp = v_new(g);
    memcpy(tmp, src, sizeof(dc) * 3 * g->V);
    s = tmp;
  }
#pragma omp parallel for
  for (long x = r.lo; x < r.hi; x++) {
    dc acc[3] = {0, 0, 0};
    for (int i = 0; i < f->nlinks; i++) {
      long y = nbr(g, x, f->dbl_mu[i], f->dbl_disp[i]);
      mv_mul_acc(acc, f->dbl[i] + 9 * x, s + 3 * y);
    }
    for (int c = 0; c < 3; c++) dest[3 * x + c] = acc[c];
  }
  free(tmp);
}

/* out = mass*in (+ sum) on subset (asqtad_dslash_p.c:1019-1023) */
static void mass_term(const or_lat *g, dc *out, const dc *in, double mass,
                      const dc *sum, int eo) {
  rng r = R(g, eo);
  if (!sum) { VLOOP(r) out[e] = mass * in[e]; }
  else { VLOOP(r) out[e] = mass * in[e] + sum[e]; }
}

void or_dslash(or_fla *f, double mass, double *outr, const double *inr,
               int eo_out, int eo_in) {
  dc *out = (dc *)outr;
  const dc *in = (const dc *)inr;
  const or_lat *g = f->g;
  if (eo_in == eo_out) {
    if (eo_out == EVENODD) { hop(f, out, in, EVENODD); mass_term(g, out, in, mass, out, EVENODD); }
    else mass_term(g, out, in, mass, NULL, eo_out);
    return;
  }
  if (eo_out == EVEN || eo_out == EVENODD) {
    if (eo_in == ODD) hop(f, out, in, EVEN);
    else if (eo_in == EVEN) mass_term(g, out, in, mass, NULL, EVEN);
    else { hop(f, out, in, EVEN); mass_term(g, out, in, mass, out, EVEN); }
  }
  if (eo_out == ODD || eo_out == EVENODD) {
    if (eo_in == EVEN) hop(f, out, in, ODD);
    else if (eo_in == ODD) mass_term(g, out, in, mass, NULL, ODD);
    else { hop(f, out, in, ODD); mass_term(g, out, in, mass, out, ODD); }
  }
}

/* one direction, accumulating (asqtad_dslash_p.c:1166-1191, style 1) */
void or_dslash_dir(or_fla *f, int dir, int fb, double wtfat, double wtlong,
                   double *outr, const double *inr, int eo_out) {
  dc *out = (dc *)outr;
  const dc *in = (const dc *)inr;
  const or_lat *g = f->g;
  rng r = R(g, eo_out);
  int i0, n = 2;
  if (f->nlinks == 16) i0 = fb > 0 ? 4 * dir : 4 * dir + 2;
  else { i0 = fb > 0 ? 2 * dir : 2 * dir + 1; n = 1; }
  double wt[2] = {wtfat, wtlong};
  const dc *src = in;
  dc *tmp = NULL;
  if (out == in) { tmp = v_new(g); memcpy(tmp, in, sizeof(dc) * 3 * g->V); src = tmp; }
#pragma omp parallel for
  for (long x = r.lo; x < r.hi; x++) {
    for (int k = 0; k < n; k++) {
      int i = i0 + k;
      long y = nbr(g, x, f->dbl_mu[i], f->dbl_disp[i]);
      dc v[3] = {wt[k] * src[3 * y], wt[k] * src[3 * y + 1], wt[k] * src[3 * y + 2]};
      mv_mul_acc(out + 3 * x, f->dbl[i] + 9 * x, v);
    }
  }
  free(tmp);
}

/* asqtad_dslash_p.c:1106-1138 */
static double ddagd_impl(or_fla *f, double mass, dc *out, const dc *in, int eo, int want_norm) {
  const or_lat *g = f->g;
  dc *tmp = v_new(g);
  double m2 = mass * mass;
  or_dslash(f, mass, (double *)tmp, (const double *)in, opp(eo), eo);
  or_dslash(f, mass, (double *)out, (const double *)tmp, eo, opp(eo));
  rng r = R(g, eo);
  VLOOP(r) out[e] = m2 * in[e] - out[e];
  double res = 0;
  if (want_norm) res = v_norm2(tmp, R(g, opp(eo))) + m2 * v_norm2(in, r);
  free(tmp);
  return res;
}
void or_ddagd(or_fla *f, double mass, double *out, const double *in, int eo) {
  ddagd_impl(f, mass, (dc *)out, (const dc *)in, eo, 0);
}
double or_ddagd_norm2(or_fla *f, double mass, double *out, const double *in, int eo) {
  return ddagd_impl(f, mass, (dc *)out, (const dc *)in, eo, 1);
}

/* examples/asqtad_test.c:37-81 (check_op), rebuilt independently from the
   unscaled links with plain neighbour gathers */
double or_check_op(or_fla *f, double mass, const double *inr, double *fatr[4], double *lngr[4]) {
  const or_lat *g = f->g;
  const dc *in = (const dc *)inr;
  dc *out = v_new(g), *chk = v_new(g);
  or_dslash(f, mass, (double *)out, inr, EVENODD, EVENODD);
#pragma omp parallel for
  for (long x = 0; x < g->V; x++) {
    dc acc[3];
    for (int c = 0; c < 3; c++) acc[c] = 2 * mass * in[3 * x + c];
    for (int mu = 0; mu < 4; mu++) {
      const dc *F = (const dc *)fatr[mu];
      dc t[3];
      mv_mul_acc(acc, F + 9 * x, in + 3 * nbr(g, x, mu, 1));
      long y = nbr(g, x, mu, -1);
      mav_mul(t, F + 9 * y, in + 3 * y);
      for (int c = 0; c < 3; c++) acc[c] -= t[c];
      if (lngr) {
        const dc *Lm = (const dc *)lngr[mu];
        mv_mul_acc(acc, Lm + 9 * x, in + 3 * nbr(g, x, mu, 3));
        long y3 = nbr(g, x, mu, -3);
        mav_mul(t, Lm + 9 * y3, in + 3 * y3);
        for (int c = 0; c < 3; c++) acc[c] -= t[c];
      }
    }
    for (int c = 0; c < 3; c++) chk[3 * x + c] = 0.5 * acc[c] - out[3 * x + c];
  }
  rng all = R(g, EVENODD);
  double d2 = v_norm2(chk, all) / v_norm2(in, all);
  free(out); free(chk);
  return d2;
}

/* ------------------------------------------------------------------ */
/* solvers: lib/invert_cg_p.c                                           */
/* ------------------------------------------------------------------ */
typedef struct { or_fla *f; double mass; int eo; } linop_ctx;

static void lin_d2(linop_ctx *L, dc *out, const dc *in) { or_ddagd(L->f, L->mass, (double *)out, (const double *)in, L->eo); }
static double lin_d2n(linop_ctx *L, dc *out, const dc *in) { return or_ddagd_norm2(L->f, L->mass, (double *)out, (const double *)in, L->eo); }

/* restarted CG: invert_cg_p.c:1-128 */
static void cg(linop_ctx *L, or_invert_arg *ia, or_resid_arg *ra, dc *out, const dc *in,
               dc *p, int eo) {
  const or_lat *g = L->f->g;
  rng r_ = R(g, eo);
  int iteration = 0, total = 0, nrestart = -1;
  int restart_it = ia->restart, max_it = ia->max_iter, max_restarts = ia->max_restarts;
  if (max_restarts < 0) max_restarts = 5;
  ra->final_rsq = 0; ra->final_rel = 0; ra->final_iter = 0; ra->final_restart = 0;
  double insq = v_norm2(in, r_);
  if (insq == 0.) { v_zero(out, r_); return; }
  dc *r = v_new(g), *Mp = v_new(g);
  double rsqstop = ra->rsqmin * insq, rsq = 0, oldrsq, relnorm2 = 1, a, b, pkp;
  oldrsq = rsq;
  while (1) {
    if (total == 0 || iteration >= restart_it || total >= max_it || rsq < rsqstop || relnorm2 < ra->relmin) {
      if (total >= max_it || nrestart >= max_restarts) break;
      nrestart++;
      v_copy(p, out, r_);
      lin_d2(L, Mp, p);
      iteration = 1; total++;
      VLOOP(r_) r[e] = in[e] - Mp[e];
      rsq = v_norm2(r, r_);
      if (ra->relmin > 0) relnorm2 = or_relnorm2(g, (double *)r, (double *)out, eo);
      if (rsq < rsqstop || relnorm2 < ra->relmin || total >= max_it) break;
      v_copy(p, r, r_);
    } else {
      b = rsq / oldrsq;
      VLOOP(r_) p[e] = b * p[e] + r[e];
    }
    oldrsq = rsq;
    lin_d2(L, Mp, p);
    iteration++; total++;
    pkp = v_redot(p, Mp, r_);
    if (pkp <= 0) break;
    a = rsq / pkp;
    VLOOP(r_) { out[e] += a * p[e]; r[e] -= a * Mp[e]; }
    rsq = v_norm2(r, r_);
    if (ra->relmin > 0) relnorm2 = or_relnorm2(g, (double *)r, (double *)out, eo);
  }
  free(r); free(Mp);
  ra->final_rsq = rsq / insq;
  ra->final_rel = relnorm2;
  ra->final_iter = total;
  ra->final_restart = nrestart;
}

/* multi-shift CG: invert_cg_p.c:130-402 */
static void cgms(linop_ctx *L, or_invert_arg *ia, or_resid_arg **ra, const double *shifts,
                 int ns, dc **out, const dc *in, dc *p, int eo) {
  const or_lat *g = L->f->g;
  rng q = R(g, eo);
  double a[ns], b[ns], bo[ns], z[ns], zo[ns], zn[ns];
  double insq = v_norm2(in, q);
  if (insq == 0.) {
    for (int i = 0; i < ns; i++) {
      v_zero(out[i], q);
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
  double rsqstop = ra[irsq]->rsqmin * insq, relstop = ra[irel]->relmin;
  dc *r = v_new(g), *Mp = v_new(g), *pm[ns];
  v_copy(r, in, q);
  for (int i = 0; i < ns; i++) {
    pm[i] = (i == imin) ? p : v_new(g);
    v_zero(out[i], q);
    v_copy(pm[i], r, q);
    zo[i] = z[i] = 1; bo[i] = -1; a[i] = 0; b[i] = 0; zn[i] = 1;
  }
  double rsq = insq, oldrsq, relnorm2 = 1, trueRsqFac = 1, trueRelFac = 1, yAy = 0;
  const int rsqCheckInterval = 100, relCheckInterval = 100;
  int nextRsqCheck = rsqCheckInterval, nextRelCheck = relCheckInterval;
  dc *y = v_new(g), *Ay = v_new(g), *ry = v_new(g);
  v_copy(ry, in, q);
  while (1) {
    oldrsq = rsq;
    double pkp = lin_d2n(L, Mp, p);
    iteration++;
    if (pkp <= 0) break;
    b[imin] = rsq / pkp;
    { double bb = b[imin]; VLOOP(q) { out[imin][e] += bb * p[e]; r[e] -= bb * Mp[e]; } }
    zn[imin] = 1;
    for (int i = 0; i < ns; i++) {
      if (i == imin) continue;
      zn[i] = z[i] * zo[i] * bo[imin];
      double c1 = b[imin] * a[imin] * (zo[i] - z[i]);
      c1 += zo[i] * bo[imin] * (1 + shifts[i] * b[imin]);
      if (c1 != 0.0) zn[i] /= c1; else zn[i] = 0;
      if (z[i] != 0.0) b[i] = b[imin] * zn[i] / z[i]; else zn[i] = b[i] = 0;
    }
    for (int i = 0; i < ns; i++) {
      if (i == imin) continue;
      double bb = b[i]; dc *o = out[i], *pp = pm[i];
      VLOOP(q) o[e] += bb * pp[e];
    }
    rsq = v_norm2(r, q);
    double rsqc = zn[irsq] * zn[irsq] * rsq;
    if (relstop > 0) relnorm2 = zn[irel] * zn[irel] * or_relnorm2(g, (double *)r, (double *)out[irel], eo);
    if (iteration >= ia->restart || iteration >= ia->max_iter) break;
    if (rsqc * trueRsqFac < rsqstop) nextRsqCheck = iteration;
    if (relnorm2 * trueRelFac < relstop) nextRelCheck = iteration;
    if (nextRsqCheck <= iteration || (relstop > 0 && nextRelCheck <= iteration)) {
      if (yAy > 0) {
        dc c = v_dot(Ay, out[imin], q) / (-yAy);
        dc *o = out[imin];
        VLOOP(q) o[e] += c * y[e];
      }
      double xAx = lin_d2n(L, Mp, out[imin]);
      iteration++;
      if (xAx <= 0) break;
      dc c = v_dot(out[imin], ry, q) / xAx;
      { dc *o = out[imin]; VLOOP(q) y[e] += c * o[e]; }
      yAy = lin_d2n(L, Ay, y);
      iteration++;
      VLOOP(q) ry[e] = in[e] - Ay[e];
      v_zero(out[imin], q);
    }
    if (nextRsqCheck <= iteration) {
      double tr2;
      if (irsq == imin) {
        tr2 = v_norm2(ry, q);
      } else {
        double xAx = lin_d2n(L, Mp, out[irsq]);
        iteration++;
        if (xAx <= 0) break;
        VLOOP(q) Mp[e] -= in[e];
        tr2 = v_norm2(Mp, q);
      }
      if (tr2 <= rsqstop) { rsq = tr2; break; }
      if (tr2 > 2 * rsq) break;
      trueRsqFac = tr2 / rsq;
      nextRsqCheck += rsqCheckInterval;
    }
    if (relstop > 0 && nextRelCheck <= iteration) {
      double xAx = lin_d2n(L, Mp, out[irel]);
      iteration++;
      if (xAx <= 0) break;
      VLOOP(q) Mp[e] -= in[e];
      double rel2 = or_relnorm2(g, (double *)Mp, (double *)out[irel], eo);
      if (rel2 <= relstop) { relnorm2 = rel2; break; }
      trueRelFac = rel2 / relnorm2;
      nextRelCheck += relCheckInterval;
      relnorm2 = rel2;
    }
    a[imin] = rsq / oldrsq;
    { double aa = a[imin]; VLOOP(q) p[e] = aa * p[e] + r[e]; }
    for (int i = 0; i < ns; i++) {
      if (i == imin) continue;
      double c2 = z[i] * b[imin];
      a[i] = (c2 != 0.0) ? a[imin] * zn[i] * b[i] / c2 : 0;
    }
    for (int i = 0; i < ns; i++) {
      if (i == imin) continue;
      double ai = a[i], zi = zn[i]; dc *pp = pm[i];
      VLOOP(q) pp[e] = ai * pp[e] + zi * r[e];
    }
    for (int i = 0; i < ns; i++) { bo[i] = b[i]; zo[i] = z[i]; z[i] = zn[i]; }
  }
  v_copy(out[imin], y, q);
  free(y); free(Ay); free(ry); free(r); free(Mp);
  for (int i = 0; i < ns; i++) if (i != imin) free(pm[i]);
  for (int i = 0; i < ns; i++) {
    double s = zn[i] * zn[i];
    ra[i]->final_rsq = s * trueRsqFac * rsq / insq;
    ra[i]->final_rel = s * trueRelFac * relnorm2;
    ra[i]->final_iter = iteration;
    ra[i]->final_restart = 0;
  }
}

/* ------------------------------------------------------------------ */
/* drivers: lib/asqtad_invert_p.c                                       */
/* ------------------------------------------------------------------ */
static double nflop_per_site(const or_fla *f) { return 0.5 * (20 * 3 + 2 * 8 * 3 * 3 * f->nlinks); }

/* refine: asqtad_invert_p.c:246-330.  r[i] on opsub holds A out[i]; the
   final residual r = in + scale*(D_ab D_ba out - m^2 out) lands on insub. */
static void refine(or_fla *f, dc **out, dc **in, dc **r, double *r2, const double *m2,
                   dc *scale, int no, int ineo, dc **x, dc **Ax, int nx,
                   const int *oi, const int *xi, int ni, dc *tv) {
  const or_lat *g = f->g;
  int opeo = opp(ineo);
  rng is = R(g, ineo), os = R(g, opeo);
  dc **Aout = r;
  for (int i = 0; i < nx; i++) or_dslash(f, 0, (double *)Ax[i], (double *)x[i], opeo, ineo);
  double x2[nx + 1], Ax2[nx + 1];
  for (int i = 0; i < nx; i++) { x2[i] = v_norm2(x[i], is); Ax2[i] = v_norm2(Ax[i], os); }
  for (int i = 0; i < ni; i++) {
    int ko = oi[i], kx = nx > 0 ? xi[i] : 0;
    dc z, Az, s, sx = 0;
    double d = 0;
    or_dslash(f, 0, (double *)Aout[ko], (double *)out[ko], opeo, ineo);
    if (nx > 0) {
      z = v_dot(x[kx], out[ko], is);
      Az = v_dot(Ax[kx], Aout[ko], os);
      d = Ax2[kx] + m2[ko] * x2[kx];
    }
    if (d != 0) {
      double di = 1 / d, dim2 = di * m2[ko];
      s = dim2 * z + di * Az;
      { dc *o = out[ko], *xx = x[kx]; VLOOP(is) o[e] -= s * xx[e]; }
      { dc *o = Aout[ko], *xx = Ax[kx]; VLOOP(os) o[e] -= s * xx[e]; }
      z = v_dot(x[kx], in[ko], is);
      sx = di * z;
    }
    z = v_dot(out[ko], in[ko], is);
    double o2 = v_norm2(out[ko], is), Ao2 = v_norm2(Aout[ko], os);
    d = Ao2 + m2[kx] * o2;      /* the reference indexes m2 by kx here */
    if (d != 0) {
      double di = 1 / d;
      s = di * z;
      scale[ko] = s;
      if (nx > 0) {
        dc zz = sx / s;
        { dc *o = out[ko], *xx = x[kx]; VLOOP(is) o[e] += zz * xx[e]; }
        { dc *o = Aout[ko], *xx = Ax[kx]; VLOOP(os) o[e] += zz * xx[e]; }
      }
    } else {
      scale[ko] = sx;
      if (nx > 0) { v_copy(out[ko], x[kx], is); v_copy(Aout[ko], Ax[kx], os); }
    }
  }
  for (int i = 0; i < no; i++) {
    or_dslash(f, 0, (double *)tv, (double *)Aout[i], ineo, opeo);
    double mm = m2[i];
    dc sc = scale[i], *o = out[i], *rr = r[i], *ii = in[i];
    VLOOP(is) { tv[e] -= mm * o[e]; rr[e] = sc * tv[e] + ii[e]; }
    r2[i] = v_norm2(r[i], is);
  }
}

/* asqtad_invert_p.c:332-647 */
void or_solve_multi(or_fla *f, or_invert_arg *ia, or_resid_arg *ra[], double masses[],
                    double *outr[], double *inr[], int nsolve, double *final_flop) {
  const or_lat *g = f->g;
  int ineo = ia->evenodd;
  if (ineo == EVENODD) {
    double fl = 0, t;
    for (int i = 0; i < nsolve; i++) {
      or_invert(f, ia, ra[i], masses[i], outr[i], inr[i], &t);
      fl = t;
    }
    if (final_flop) *final_flop = fl;
    return;
  }
  dc **out = (dc **)outr, **in = (dc **)inr;
  rng is = R(g, ineo);
  int opeo = opp(ineo);
  dc *tv = v_new(g), *r[nsolve], scale[nsolve];
  double in2[nsolve], r2[nsolve], r2stop[nsolve], mass2[nsolve], m2s[nsolve];
  int oi[nsolve], xi[nsolve], nm = 0, iter = 0, nrestart = -1;
  int max_iter = ia->max_iter, max_restarts = ia->max_restarts;
  double mixedrsq = ia->mixed_rsq;
  dc *cgp = v_new(g);
  for (int i = 0; i < nsolve; i++) in2[i] = v_norm2(in[i], is);
  for (int i = 0; i < nsolve; i++) {
    r2stop[i] = ra[i]->rsqmin * in2[i];
    mass2[i] = masses[i] * masses[i];
    oi[i] = i;
    int j = nm;
    while (j > 0 && mass2[i] < m2s[j - 1]) j--;
    if (j == nm || m2s[j] != mass2[i]) {
      for (int k = nm; k > j; k--) m2s[k] = m2s[k - 1];
      m2s[j] = mass2[i];
      nm++;
    }
    r[i] = v_new(g);
    or_dslash(f, 0, (double *)r[i], (double *)out[i], opeo, ineo);
  }
  for (int i = 0; i < nsolve; i++) {
    int j = 0;
    while (j < nm - 1 && m2s[j] != mass2[i]) j++;
    xi[i] = j;
  }
  or_resid_arg resarg0 = {0, 0, 0, 0, 0, 0};
  or_resid_arg *xresarg[nm];
  dc *x[nm];
  double m20 = m2s[0];
  linop_ctx L = {f, sqrt(m20), ineo};
  for (int i = 0; i < nm; i++) { m2s[i] -= m20; x[i] = v_new(g); }
  refine(f, out, in, r, r2, mass2, scale, nsolve, ineo, NULL, NULL, 0, oi, NULL, nsolve, tv);
  while (1) {
    for (int i = 0; i < nsolve; i++)
      ra[i]->final_rel = ra[i]->relmin > 0 ? or_relnorm2(g, (double *)r[i], (double *)out[i], ineo) : 1;
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
    }
    if (r2max <= r2stopmax || nrestart >= max_restarts || iter >= max_iter) break;
    for (int i = 0; i < nm; i++) {
      xresarg[i] = (i == xi[imax]) ? ra[imax] : &resarg0;
      memset(x[i], 0, sizeof(dc) * 3 * g->V);
    }
    double rsqminold = ra[imax]->rsqmin;
    ra[imax]->rsqmin = r2stopmax / r2max;
    if (ra[imax]->rsqmin >= 1) ra[imax]->rsqmin = in2max * r2stopmax / r2max;
    ra[imax]->rsqmin *= rsqminfac;
    ia->max_iter = max_iter - iter;
    /* double-precision build: the inner solve runs in single precision
       when r2max > mixed_rsq*in2max (:510-537); the oracle keeps FP64 but
       reproduces the changed inner tolerance */
    if (r2max > mixedrsq * in2max && mixedrsq > rsqminold) ra[imax]->rsqmin = mixedrsq * in2max / r2max;
    cgms(&L, ia, xresarg, m2s, nm, x, r[imax], cgp, ineo);
    iter += ra[imax]->final_iter;
    nrestart++;
    ra[imax]->rsqmin = rsqminold;
    if (usingrel) {
      for (int i = 0; i < nsolve; i++) {
        int ko = oi[i], kx = xi[i];
        double s2 = creal(scale[ko]) * creal(scale[ko]) + cimag(scale[ko]) * cimag(scale[ko]);
        if (s2 == 0.0) v_copy(out[ko], x[kx], is);
        else { dc s = 1.0 / scale[ko]; dc *o = out[ko], *xx = x[kx]; VLOOP(is) o[e] += s * xx[e]; }
      }
      refine(f, out, in, r, r2, mass2, scale, nsolve, ineo, NULL, NULL, 0, oi, NULL, nsolve, tv);
    } else {
      refine(f, out, in, r, r2, mass2, scale, nsolve, ineo, x, x, nm, oi, xi, nsolve, tv);
    }
  }
  ia->max_iter = max_iter;
  for (int i = 0; i < nsolve; i++) {
    dc s = masses[i] * scale[i];
    dc *o = out[i];
    VLOOP(is) o[e] = s * o[e];
    ra[i]->final_iter = iter;
    ra[i]->final_rsq = in2[i] > 0 ? r2[i] / in2[i] : 0;
    ra[i]->final_restart = nrestart > 0 ? nrestart : 0;
  }
  if (final_flop) *final_flop = (nflop_per_site(f) + 0.5 * 10 * 3 * (nm - 1)) * iter * g->V;
  for (int i = 0; i < nm; i++) free(x[i]);
  for (int i = 0; i < nsolve; i++) free(r[i]);
  free(tv); free(cgp);
}

/* asqtad_invert_p.c:649-851 */
void or_invert(or_fla *f, or_invert_arg *ia, or_resid_arg *ra, double mass,
               double *outr, const double *inr, double *final_flop) {
  if (ia->evenodd != EVENODD) {
    double *o[1] = {outr}, *i_[1] = {(double *)inr}, m[1] = {mass};
    or_resid_arg *rr[1] = {ra};
    or_solve_multi(f, ia, rr, m, o, i_, 1, final_flop);
    return;
  }
  const or_lat *g = f->g;
  dc *out = (dc *)outr;
  const dc *in = (const dc *)inr;
  int iter = 0, max_iter_old = ia->max_iter, max_restarts_old = ia->max_restarts;
  int nrestart = -1, max_restarts = ia->max_restarts;
  if (max_restarts <= 0) max_restarts = 5;
  int ineo = ia->evenodd;
  rng is = R(g, ineo);
  double insqe = 0, insqo = 0;
  if (ineo != ODD) insqe = v_norm2(in, R(g, EVEN));
  if (ineo != EVEN) insqo = v_norm2(in, R(g, ODD));
  double insq = insqe + insqo;
  int cgeo = insqe >= insqo ? EVEN : ODD;
  rng cs = R(g, cgeo), ocs = R(g, opp(cgeo));
  linop_ctx L = {f, mass, cgeo};
  dc *cgp = v_new(g), *cgr = v_new(g), *tmp2 = v_new(g), *qin = v_new(g), *qout = v_new(g);
  v_copy(tmp2, in, is);
  /* project: qin_cg = mass*in_cg - D_cg,opp in_opp (:80-89) */
  or_dslash(f, mass, (double *)qin, (double *)tmp2, cgeo, opp(cgeo));
  VLOOP(cs) qin[e] = mass * tmp2[e] - qin[e];
  if (ineo == cgeo) v_zero(qin, ocs); else v_copy(qin, in, ocs);
  double pinsq = v_norm2(qin, cs);
  double rsqfac = mass * mass * insq / pinsq;
  v_copy(qout, out, cs);
  double rsqstop = insq * ra->rsqmin, rsq = 0, relnorm2 = 1.;
  double rsqminold = ra->rsqmin, relminold = ra->relmin;
  ra->rsqmin = 0.99 * rsqminold * rsqfac;
  ra->relmin = 0.99 * relminold;
  ia->max_restarts = 0;
  do {
    cg(&L, ia, ra, qout, qin, cgp, cgeo);
    iter += ra->final_iter;
    /* reconstruct (:92-100): out_opp = (src_opp - D_opp,cg soln_cg)/mass */
    v_copy(cgr, qout, cs);
    or_dslash(f, mass, (double *)qout, (double *)cgr, opp(cgeo), cgeo);
    VLOOP(ocs) qout[e] = (qin[e] - qout[e]) * (1.0 / mass);
    or_dslash(f, mass, (double *)cgr, (double *)qout, ineo, EVENODD);
    VLOOP(is) cgr[e] -= in[e];
    rsq = v_norm2(cgr, is);
    ra->rsqmin *= 0.99;
    if (ra->relmin > 0) {
      relnorm2 = or_relnorm2(g, (double *)cgr, (double *)qout, ineo);
      ra->relmin = 0.99 * ra->final_rel / relnorm2 * relminold;
    }
    ia->max_iter = max_iter_old - iter;
  } while ((++nrestart < max_restarts) && (ia->max_iter > 0) && (rsq > rsqstop) && (relnorm2 > ra->relmin));
  v_copy(out, qout, is);
  ia->max_iter = max_iter_old;
  ia->max_restarts = max_restarts_old;
  ra->rsqmin = rsqminold;
  ra->relmin = relminold;
  ra->final_iter = iter;
  ra->final_rsq = insq == 0. ? 0 : rsq / insq;
  ra->final_rel = relnorm2;
  ra->final_restart = nrestart;
  if (final_flop) *final_flop = nflop_per_site(f) * iter * g->V;
  free(cgp); free(cgr); free(tmp2); free(qin); free(qout);
}

/* asqtad_invert_p.c:878-1059 */
void or_invert_multi(or_fla *f, or_invert_arg *ia, or_resid_arg **ra[], double *masses[],
                     int nmass[], double **outr[], double *inr[], int nsrc, double *final_flop) {
  const or_lat *g = f->g;
  if (ia->evenodd != EVENODD) {
    int nsolve = 0;
    for (int i = 0; i < nsrc; i++) nsolve += nmass[i];
    or_resid_arg *rr[nsolve];
    double ms[nsolve], *o[nsolve], *in_[nsolve];
    int k = 0;
    for (int i = 0; i < nsrc; i++)
      for (int j = 0; j < nmass[i]; j++) { rr[k] = ra[i][j]; ms[k] = masses[i][j]; o[k] = outr[i][j]; in_[k] = inr[i]; k++; }
    or_solve_multi(f, ia, rr, ms, o, in_, nsolve, final_flop);
    return;
  }
  double nflop = nflop_per_site(f), nflopm = 0.5 * 10 * 3, flop = 0;
  int cgeo = EVEN;                  /* EVENODD is solved on the even subset */
  rng cs = R(g, cgeo);
  dc *cgp = v_new(g);
  if (nsrc == 2 && nmass[0] == 1 && nmass[1] == 1 && masses[0][0] != masses[1][0]) {
    double shifts[2], rsq0, rsq1, rsqsave[2];
    int imin = 0;
    dc *x0 = v_new(g), *src = v_new(g), *incv[2], *outcv[2];
    or_resid_arg *rr[2];
    for (int i = 0; i < 2; i++) {
      shifts[i] = masses[i][0] * masses[i][0];
      if (shifts[i] < shifts[imin]) imin = i;
      incv[i] = (dc *)inr[i]; outcv[i] = (dc *)outr[i][0]; rr[i] = ra[i][0];
    }
    double gm = masses[imin][0];
    for (int i = 0; i < 2; i++) shifts[i] -= gm * gm;
    double st = 1 / (shifts[1] - shifts[0]);
    VLOOP(cs) x0[e] = st * (incv[1][e] - incv[0][e]);
    v_copy(cgp, x0, cs);
    linop_ctx L = {f, gm, cgeo};
    lin_d2(&L, src, cgp);
    VLOOP(cs) src[e] = incv[imin][e] - src[e];
    rsq1 = v_norm2(src, cs);
    for (int i = 0; i < 2; i++) {
      rsq0 = v_norm2(incv[i], cs);
      rsqsave[i] = ra[i][0]->rsqmin;
      ra[i][0]->rsqmin *= rsq0 / rsq1;
    }
    cgms(&L, ia, rr, shifts, 2, outcv, src, cgp, cgeo);
    flop += (nflop + nflopm) * rr[imin]->final_iter * g->V;
    for (int i = 0; i < 2; i++) {
      ra[i][0]->rsqmin = rsqsave[i];
      dc *o = outcv[i];
      VLOOP(cs) o[e] += x0[e];
    }
    free(x0); free(src);
  } else {
    for (int i = 0; i < nsrc; i++) {
      double shifts[nmass[i]];
      dc *cv[nmass[i]];
      int jmin = 0;
      for (int j = 0; j < nmass[i]; j++) {
        shifts[j] = masses[i][j] * masses[i][j];
        if (shifts[j] < shifts[jmin]) jmin = j;
        cv[j] = (dc *)outr[i][j];
      }
      double gm = masses[i][jmin];
      for (int j = 0; j < nmass[i]; j++) shifts[j] -= gm * gm;
      linop_ctx L = {f, gm, cgeo};
      cgms(&L, ia, ra[i], shifts, nmass[i], cv, (dc *)inr[i], cgp, cgeo);
      flop += (nflop + nflopm * (nmass[i] - 1)) * ra[i][0]->final_iter * g->V;
    }
  }
  for (int i = 0; i < nsrc; i++)
    for (int j = 0; j < nmass[i]; j++) {
      double m = masses[i][j];
      dc *o = (dc *)outr[i][j];
      VLOOP(cs) o[e] = m * o[e];
    }
  if (final_flop) *final_flop = flop;
  free(cgp);
}

/* ------------------------------------------------------------------ */
/* asqtad fermion force: lib/asqtad_force_p.c:16-64 (entry points),     */
/* lib/asqtad_force_fnmat_p.c:4-43 (outer products, scale -1), :491-513 */
/* (sign flip on odd sites), :516-546 (force += -2 antiherm(U deriv^+)). */
/* The derivative of the smeared links is formed here by reverse-mode    */
/* differentiation of make_imp_links' staple sums (the adjoint of every  */
/* staple application, in reverse order); the reference forms the same   */
/* derivative with its staple / side-force recursion (:85-359).          */
/* ------------------------------------------------------------------ */
static inline void m_acc(dc *r, const dc *a, double c) { for (int e = 0; e < 9; e++) r[e] += c * a[e]; }

/* adjoint of fl += coef*staple(in; mu, nu) with respect to `in`:
   Gin(z) += coef [U_nu(z-nu)^+ G(z-nu) U_nu(z-nu+mu) + U_nu(z) G(z+nu) U_nu(z+mu)^+] */
static void adj_staple_in(const or_lat *g, dc *Gin, const dc *G, int mu, int nu, double coef, dc **U) {
#pragma omp parallel for
  for (long z = 0; z < g->V; z++) {
    dc t[9], r[9];
    long zmn = nbr(g, z, nu, -1), zmnpm = nbr(g, zmn, mu, 1);
    long zpn = nbr(g, z, nu, 1), zpm = nbr(g, z, mu, 1);
    m_mul_an(t, U[nu] + 9 * zmn, G + 9 * zmn);
    m_mul(r, t, U[nu] + 9 * zmnpm);
    m_acc(Gin + 9 * z, r, coef);
    m_mul(t, U[nu] + 9 * z, G + 9 * zpn);
    m_mul_na(r, t, U[nu] + 9 * zpm);
    m_acc(Gin + 9 * z, r, coef);
  }
}

/* adjoint of fl += coef*staple(in; mu, nu) with respect to U_nu:
   GU(z) += coef [G(z) U(z+mu) in(z+nu)^+ + G(z-mu)^+ U(z-mu) in(z-mu+nu)
                  + in(z-mu)^+ U(z-mu) G(z-mu+nu) + in(z) U(z+mu) G(z+nu)^+],  U = U_nu */
static void adj_staple_link(const or_lat *g, dc *GU, const dc *G, const dc *in, int mu, int nu, double coef,
                            dc **U) {
#pragma omp parallel for
  for (long z = 0; z < g->V; z++) {
    dc t[9], r[9];
    long zpm = nbr(g, z, mu, 1), zpn = nbr(g, z, nu, 1);
    long zmm = nbr(g, z, mu, -1), zmmpn = nbr(g, zmm, nu, 1);
    const dc *Un = U[nu];
    m_mul(t, G + 9 * z, Un + 9 * zpm);      m_mul_na(r, t, in + 9 * zpn);   m_acc(GU + 9 * z, r, coef);
    m_mul_an(t, G + 9 * zmm, Un + 9 * zmm); m_mul(r, t, in + 9 * zmmpn);    m_acc(GU + 9 * z, r, coef);
    m_mul_an(t, in + 9 * zmm, Un + 9 * zmm); m_mul(r, t, G + 9 * zmmpn);    m_acc(GU + 9 * z, r, coef);
    m_mul(t, in + 9 * z, Un + 9 * zpm);     m_mul_na(r, t, G + 9 * zpn);    m_acc(GU + 9 * z, r, coef);
  }
}

void or_asqtad_deriv(const or_lat *g, const double coef[6], double *Ur[4], double *midFr[4], double *midNr[4],
                     double *derivr[4], int lepage_rep) {
  dc *U[4], *M[4], *D[4];
  for (int i = 0; i < 4; i++) { U[i] = (dc *)Ur[i]; M[i] = (dc *)midFr[i]; D[i] = (dc *)derivr[i]; }
  const double c1 = coef[0] - 6 * coef[4], c3 = coef[1], c5 = coef[2], c7 = coef[3], cL = coef[4];
  const int have5 = c5 != 0 || c7 != 0 || cL != 0, have3 = c3 != 0 || have5;
  const size_t fsz = sizeof(dc) * 9 * g->V;
  dc *S3 = calloc(9 * g->V, sizeof(dc)), *S5 = calloc(9 * g->V, sizeof(dc));
  dc *G3 = malloc(fsz), *G5 = malloc(fsz), *junk = calloc(9 * g->V, sizeof(dc));
  for (int mu = 0; mu < 4; mu++) {

    for (long s = 0; s < 9 * g->V; s++) D[mu][s] += c1 * M[mu][s];
    if (!have3) continue;
    for (int nu = 0; nu < 4; nu++) {
      if (nu == mu) continue;
      memset(junk, 0, fsz);
      gen_staple(g, S3, mu, nu, U[mu], 0.0, U, junk);              /* S3 = staple(U_mu; mu, nu) */
      for (long s = 0; s < 9 * g->V; s++) G3[s] = c3 * M[mu][s];
      if (cL != 0) {                                                /* fl += cL staple(S3; mu, nu) */
        adj_staple_in(g, G3, M[mu], mu, nu, cL, U);
        adj_staple_link(g, D[nu], M[mu], S3, mu, nu, cL, U);
      }
      if (c5 != 0 || c7 != 0) {
        for (int rho = 0; rho < 4; rho++) {
          if (rho == mu || rho == nu) continue;
          memset(junk, 0, fsz);
          gen_staple(g, S5, mu, rho, S3, 0.0, U, junk);           /* S5 = staple(S3; mu, rho) */
          for (long s = 0; s < 9 * g->V; s++) G5[s] = c5 * M[mu][s];
          if (c7 != 0)
            for (int sig = 0; sig < 4; sig++) {
              if (sig == mu || sig == nu || sig == rho) continue;   /* fl += c7 staple(S5; mu, sig) */
              adj_staple_in(g, G5, M[mu], mu, sig, c7, U);
              adj_staple_link(g, D[sig], M[mu], S5, mu, sig, c7, U);
            }
          adj_staple_in(g, G3, G5, mu, rho, 1.0, U);
          adj_staple_link(g, D[rho], G5, S3, mu, rho, 1.0, U);
        }
      }
      adj_staple_in(g, D[mu], G3, mu, nu, 1.0, U);
      adj_staple_link(g, D[nu], G3, U[mu], mu, nu, 1.0, U);
    }
  }
  if (midNr && coef[5] != 0) {                                      /* long = naik U U U */
    const double cn = coef[5];
    for (int mu = 0; mu < 4; mu++) {
      const dc *N = (const dc *)midNr[mu], *Um = U[mu];
#pragma omp parallel for
      for (long z = 0; z < g->V; z++) {
        dc t[9], r[9];
        long p1 = nbr(g, z, mu, 1), p2 = nbr(g, p1, mu, 1);
        long m1 = nbr(g, z, mu, -1), m2 = nbr(g, m1, mu, -1);
        m_mul(t, Um + 9 * p1, Um + 9 * p2);   m_mul_na(r, N + 9 * z, t);       m_acc(D[mu] + 9 * z, r, cn);
        m_mul_an(t, Um + 9 * m1, N + 9 * m1); m_mul_na(r, t, Um + 9 * p1);     m_acc(D[mu] + 9 * z, r, cn);
        m_mul(t, Um + 9 * m2, Um + 9 * m1);   m_mul_an(r, t, N + 9 * m2);      m_acc(D[mu] + 9 * z, r, cn);
      }
    }
  }
  /* lepage_rep: with a Lepage term the reference's derivative field carries
     one more term, of the form U_mu H with H Hermitian
     (lib/asqtad_force_fnmat_p.c:316-340):
     D_mu(x) -= cL [F_mu(x) U_mu(x) - U_mu(x) F_mu(x+mu)],
     F_mu = sum_{nu != mu} (A_nu + A_nu^+),
     A_nu(x) = M_nu(x) U_nu(x)^+ - M_nu(x-nu)^+ U_nu(x-nu).
     The force projection TA(U D^+) removes it; the filtered U(3) adjoint of
     the HISQ force, which receives this field at the W level, does not. */
  if (lepage_rep && cL != 0) {
    dc *Hn = calloc(4 * 9 * (size_t)g->V, sizeof(dc));
    for (int nu = 0; nu < 4; nu++)
#pragma omp parallel for
      for (long z = 0; z < g->V; z++) {
        dc a[9], b[9];
        long zm = nbr(g, z, nu, -1);
        m_mul_na(a, M[nu] + 9 * z, U[nu] + 9 * z);
        m_mul_an(b, M[nu] + 9 * zm, U[nu] + 9 * zm);
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) {
            dc aij = a[3 * i + j] - b[3 * i + j], aji = a[3 * j + i] - b[3 * j + i];
            Hn[9 * (nu * g->V + z) + 3 * i + j] = aij + conj(aji);
          }
      }
    for (int mu = 0; mu < 4; mu++)
#pragma omp parallel for
      for (long z = 0; z < g->V; z++) {
        dc F0[9] = {0}, F1[9] = {0}, r[9], t[9];
        long zp = nbr(g, z, mu, 1);
        for (int nu = 0; nu < 4; nu++) {
          if (nu == mu) continue;
          m_acc(F0, Hn + 9 * (nu * g->V + z), 1.0);
          m_acc(F1, Hn + 9 * (nu * g->V + zp), 1.0);
        }
        m_mul(r, F0, U[mu] + 9 * z);
        m_mul(t, U[mu] + 9 * z, F1);
        m_acc(r, t, -1.0);
        m_acc(D[mu] + 9 * z, r, -cL);
      }
    free(Hn);
  }
  free(S3); free(S5); free(G3); free(G5); free(junk);
}

void or_asqtad_force(const or_lat *g, const double coef[6], double *Ur[4], double *forcer[4], const double *eps,
                     double *xr[], int nsrc, int asvec) {
  const size_t n = 9 * (size_t)g->V;
  double *mid[8], *der[4];
  for (int i = 0; i < 8; i++) mid[i] = calloc(2 * n, sizeof(double));
  for (int i = 0; i < 4; i++) der[i] = calloc(2 * n, sizeof(double));
  for (int mu = 0; mu < 4; mu++) {
    dc *MF = (dc *)mid[mu], *MN = (dc *)mid[4 + mu];
#pragma omp parallel for
    for (long z = 0; z < g->V; z++) {
      const int *xc = g->x + 4 * z;
      const double sgn = ((xc[0] + xc[1] + xc[2] + xc[3]) & 1) ? 1.0 : -1.0;   /* -1 times (-1 on odd) */
      long z1 = nbr(g, z, mu, 1), z3 = nbr(g, z, mu, 3);
      for (int i = 0; i < nsrc; i++) {
        const dc *x = (const dc *)xr[i];
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) {
            MF[9 * z + 3 * a + b] += sgn * eps[i] * x[3 * z + a] * conj(x[3 * z1 + b]);
            MN[9 * z + 3 * a + b] += sgn * eps[i] * x[3 * z + a] * conj(x[3 * z3 + b]);
          }
      }
    }
  }
  or_asqtad_deriv(g, coef, Ur, mid, coef[5] != 0 ? mid + 4 : NULL, der, 0);
  /* FNMAT (asqtad_force_fnmat_p.c:530-540): force += -2 TA(U deriv^+).
     ASVEC (asqtad_force_asvec_p.c:180-184, 403-408; chosen by
     asqtad_force_p.c:22 when nsrc < fnmat_src_min): the outer products are
     accumulated into the force field itself and the traceless anti-Hermitian
     part of the sum is stored, force = TA(force + C); for the same inputs
     TA(C) = -TA(U deriv^+), half the FNMAT contribution (as the reference,
     compiled by oracle/ref, computes it). */
  const double fac = asvec ? -1.0 : -2.0;
  for (int mu = 0; mu < 4; mu++) {
    const dc *Um = (const dc *)Ur[mu], *Dm = (const dc *)der[mu];
    dc *F = (dc *)forcer[mu];
#pragma omp parallel for
    for (long z = 0; z < g->V; z++) {
      dc a[9], f[9];
      m_mul_na(a, Um + 9 * z, Dm + 9 * z);                 /* U deriv^+ */
      dc tr = 0, trf = 0;
      for (int k = 0; k < 3; k++) tr += a[4 * k] - conj(a[4 * k]);
      for (int e = 0; e < 9; e++) f[e] = F[9 * z + e];
      for (int k = 0; k < 3; k++) trf += f[4 * k] - conj(f[4 * k]);
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          dc ta = 0.5 * (a[3 * i + j] - conj(a[3 * j + i]));
          if (i == j) ta -= tr / 6.0;
          dc base = f[3 * i + j];
          if (asvec) {   /* TA of the incoming force */
            base = 0.5 * (f[3 * i + j] - conj(f[3 * j + i]));
            if (i == j) base -= trf / 6.0;
          }
          F[9 * z + 3 * i + j] = base + fac * ta;
        }
    }
  }
  for (int i = 0; i < 8; i++) free(mid[i]);
  for (int i = 0; i < 4; i++) free(der[i]);
}

/* ------------------------------------------------------------------ */
/* HISQ fermion force: lib/hisq_force_p.c:50-80 (n_orders_naik groups),  */
/* lib/hisq_force_fnmat2_p.c:7-162 (mid with scale +1, sign flip on odd  */
/* sites, asqtad level on W with the difference terms weighted by        */
/* eps_naik, reunitarisation, fat7 level on U, factor 2), :164-231       */
/* (force += antiherm(U deriv^+)).  The reunitarisation adjoint is the   */
/* derivative of the polar factor W = V f(Q), Q = V^+V, f(q) = q^-1/2:   */
/*   GV = GW f + V (B + B^+),  B = Z [(Z^+ V^+ GW Z) o Gamma] Z^+,        */
/*   Gamma_ij = (f(w_i) - f(w_j)) / (w_i - w_j)                           */
/*            = -1 / (s_i s_j (s_i + s_j)),  s = sqrt(w)  (i = j: f'(w)).  */
/* Force filter (lib/hisq_reunit_utilities_p.c:463-481, the option        */
/* force_filter of QOP_hisq_force_set_opts, 5e-5 by default): when the    */
/* smallest eigenvalue of Q is below ff, the derivative is the one of     */
/* V (Q + ff)^-1/2, every w shifted by ff (the projection itself is not). */
/* ------------------------------------------------------------------ */
static void reunit_adj(const dc *V, const dc *GW, dc *GV, double ff) {
  dc Q[9], Z[9], f[9], A[9], t[9], At[9], B[9], u[9];
  double w[3], s[3];
  m_mul_an(Q, V, V);
  herm_eig3(Q, w, Z);
  if (ff > 0 && fmin(w[0], fmin(w[1], w[2])) < ff)
    for (int i = 0; i < 3; i++) w[i] += ff;
  for (int i = 0; i < 3; i++) s[i] = sqrt(w[i]);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      dc acc = 0;
      for (int k = 0; k < 3; k++) acc += Z[3 * i + k] * (1.0 / s[k]) * conj(Z[3 * j + k]);
      f[3 * i + j] = acc;
    }
  m_mul_an(A, V, GW);
  m_mul_an(t, Z, A);
  m_mul(At, t, Z);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) At[3 * i + j] *= -1.0 / (s[i] * s[j] * (s[i] + s[j]));
  m_mul(t, Z, At);
  m_mul_na(B, t, Z);
  m_mul(GV, GW, f);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) t[3 * i + j] = B[3 * i + j] + conj(B[3 * j + i]);
  m_mul(u, V, t);
  for (int e = 0; e < 9; e++) GV[e] += u[e];
}

void or_hisq_deriv(const or_lat *g, const double h[18], double *U[4], int n_naiks, const double *eps_naik,
                   double **midF, double **midN, double *deriv[4]) {
  const size_t n = 18 * (size_t)g->V;
  double *Vl[4], *Wl[4], *GW[4], *tmp[4], *GV[4];
  for (int i = 0; i < 4; i++) {
    Vl[i] = calloc(n, sizeof(double)); Wl[i] = calloc(n, sizeof(double));
    GW[i] = calloc(n, sizeof(double)); tmp[i] = calloc(n, sizeof(double)); GV[i] = calloc(n, sizeof(double));
  }
  const double c7[6] = {h[0], h[1], h[2], h[3], h[13] != 0 ? h[4] : 0.0, 0.0};
  or_make_imp_links(g, c7, U, U, Vl, NULL);
  for (int i = 0; i < 4; i++)
#pragma omp parallel for
    for (long s = 0; s < g->V; s++) or_u3_un_analytic(Vl[i] + 18 * s, Wl[i] + 18 * s, h[14] != 0, h[15], h[16]);
  const double ca[6] = {h[5], h[6], h[7], h[8], h[9], h[10]}, cd[6] = {h[11], 0, 0, 0, 0, h[12]};
  for (int k = 0; k < n_naiks; k++) {
    for (int i = 0; i < 4; i++) memset(tmp[i], 0, n * sizeof(double));
    or_asqtad_deriv(g, k == 0 ? ca : cd, Wl, midF + 4 * k, midN + 4 * k, tmp, 1);
    const double c = k == 0 ? 1.0 : eps_naik[k];
    for (int i = 0; i < 4; i++)
      for (size_t e = 0; e < n; e++) GW[i][e] += c * tmp[i][e];
  }
  for (int i = 0; i < 4; i++)
#pragma omp parallel for
    for (long s = 0; s < g->V; s++)
      reunit_adj((const dc *)Vl[i] + 9 * s, (const dc *)GW[i] + 9 * s, (dc *)GV[i] + 9 * s, h[17]);
  or_asqtad_deriv(g, c7, U, GV, NULL, deriv, 0);
  for (int i = 0; i < 4; i++) { free(Vl[i]); free(Wl[i]); free(GW[i]); free(tmp[i]); free(GV[i]); }
}

void or_hisq_force(const or_lat *g, const double h[18], double *Ur[4], int n_naiks, const double *eps_naik,
                   double *forcer[4], const double *res, double *xr[], const int *n_orders_naik) {
  const size_t n = 18 * (size_t)g->V;
  double **mid = malloc(sizeof(double *) * 8 * n_naiks), *der[4];
  for (int i = 0; i < 8 * n_naiks; i++) mid[i] = calloc(n, sizeof(double));
  for (int i = 0; i < 4; i++) der[i] = calloc(n, sizeof(double));
  int nterms = 0;
  for (int k = 0; k < n_naiks; k++) nterms += n_orders_naik[k];
  int shift = 0;
  for (int k = 0; k < n_naiks; k++) {
    const int first = k == 0 ? 0 : shift, count = k == 0 ? nterms : n_orders_naik[k];
    for (int mu = 0; mu < 4; mu++) {
      dc *MF = (dc *)mid[4 * k + mu], *MN = (dc *)mid[4 * n_naiks + 4 * k + mu];
#pragma omp parallel for
      for (long z = 0; z < g->V; z++) {
        const int *xc = g->x + 4 * z;
        const double sgn = ((xc[0] + xc[1] + xc[2] + xc[3]) & 1) ? -1.0 : 1.0;
        long z1 = nbr(g, z, mu, 1), z3 = nbr(g, z, mu, 3);
        for (int i = first; i < first + count; i++) {
          const dc *x = (const dc *)xr[i];
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
              MF[9 * z + 3 * a + b] += sgn * res[i] * x[3 * z + a] * conj(x[3 * z1 + b]);
              MN[9 * z + 3 * a + b] += sgn * res[i] * x[3 * z + a] * conj(x[3 * z3 + b]);
            }
        }
      }
    }
    shift += n_orders_naik[k];
  }
  or_hisq_deriv(g, h, Ur, n_naiks, eps_naik, mid, mid + 4 * n_naiks, der);
  for (int mu = 0; mu < 4; mu++) {
    const dc *Um = (const dc *)Ur[mu], *Dm = (const dc *)der[mu];
    dc *F = (dc *)forcer[mu];
#pragma omp parallel for
    for (long z = 0; z < g->V; z++) {
      dc a[9];
      m_mul_na(a, Um + 9 * z, Dm + 9 * z);
      dc tr = 0;
      for (int k = 0; k < 3; k++) tr += a[4 * k] - conj(a[4 * k]);
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          dc ta = 0.5 * (a[3 * i + j] - conj(a[3 * j + i]));
          if (i == j) ta -= tr / 6.0;
          F[9 * z + 3 * i + j] += 2.0 * ta;
        }
    }
  }
  for (int i = 0; i < 8 * n_naiks; i++) free(mid[i]);
  free(mid);
  for (int i = 0; i < 4; i++) free(der[i]);
}
