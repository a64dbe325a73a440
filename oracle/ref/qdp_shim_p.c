/* qdp_shim_p.c -- the field operations of the single-process QDP interface
   in qdp.h for one precision (compiled with QDP_Precision 'F' and 'D'):
   test infrastructure for building the reference's asqtad path.  Every
   operation loops over the sites of its subset (contiguous in raw order),
   threaded with OpenMP as QDP's own site loops are; site arithmetic is in
   the field's precision, reductions in double. */
#define QLA_Precision QDP_Precision
#include <string.h>
#include "qdp.h"

#if QDP_Precision == 'F'
typedef float R;
#else
typedef double R;
#endif
typedef QLA_Complex C;
typedef QLA_ColorVector QV;
typedef QLA_ColorMatrix QM;

#define SHIM_PRAGMA(x) _Pragma(#x)
#define SITES_SERIAL(sub) for (int i = (sub)->start; i < (sub)->start + (sub)->len; i++)
#define SITES(sub) SHIM_PRAGMA(omp parallel for schedule(static)) SITES_SERIAL(sub)
#define SITES_SUM(sub, ...) SHIM_PRAGMA(omp parallel for schedule(static) reduction(+ : __VA_ARGS__)) SITES_SERIAL(sub)

static void *shim_alloc(size_t n) {
  void *p = calloc(1, n);
  if (!p) QDP_abort(1);
  return p;
}

QDP_ColorVector *QDP_create_V(void) {
  QDP_ColorVector *v = (QDP_ColorVector *)shim_alloc(sizeof(*v));
  v->d = (QV *)shim_alloc(sizeof(QV) * QDP_shim_V);
  return v;
}
void QDP_destroy_V(QDP_ColorVector *v) {
  if (!v) return;
  free(v->d);
  free(v);
}
QDP_ColorMatrix *QDP_create_M(void) {
  QDP_ColorMatrix *m = (QDP_ColorMatrix *)shim_alloc(sizeof(*m));
  m->d = (QM *)shim_alloc(sizeof(QM) * QDP_shim_V);
  return m;
}
void QDP_destroy_M(QDP_ColorMatrix *m) {
  if (!m) return;
  free(m->d);
  free(m);
}
QDP_Complex *QDP_create_C(void) {
  QDP_Complex *c = (QDP_Complex *)shim_alloc(sizeof(*c));
  c->d = (C *)shim_alloc(sizeof(C) * QDP_shim_V);
  return c;
}
void QDP_destroy_C(QDP_Complex *c) {
  if (!c) return;
  free(c->d);
  free(c);
}
QDP_DiracFermion *QDP_create_D(void) {
  QDP_DiracFermion *f = (QDP_DiracFermion *)shim_alloc(sizeof(*f));
  f->d = (QLA_DiracFermion *)shim_alloc(sizeof(QLA_DiracFermion) * QDP_shim_V);
  return f;
}
void QDP_destroy_D(QDP_DiracFermion *f) {
  if (!f) return;
  free(f->d);
  free(f);
}
void QDP_D_eq_D(QDP_DiracFermion *r, QDP_DiracFermion *a, QDP_Subset s) { SITES(s) r->d[i] = a->d[i]; }
void QDP_insert_D(QDP_DiracFermion *f, QLA_DiracFermion *raw, QDP_Subset s) { SITES(s) f->d[i] = raw[i]; }
void QDP_extract_D(QLA_DiracFermion *raw, QDP_DiracFermion *f, QDP_Subset s) { SITES(s) raw[i] = f->d[i]; }
QV *QDP_expose_V(QDP_ColorVector *v) { return v->d; }
void QDP_reset_V(QDP_ColorVector *v) { (void)v; }
QM *QDP_expose_M(QDP_ColorMatrix *m) { return m->d; }
void QDP_reset_M(QDP_ColorMatrix *m) { (void)m; }
void QDP_insert_V(QDP_ColorVector *v, QV *raw, QDP_Subset s) { SITES(s) v->d[i] = raw[i]; }
void QDP_extract_V(QV *raw, QDP_ColorVector *v, QDP_Subset s) { SITES(s) raw[i] = v->d[i]; }
void QDP_insert_M(QDP_ColorMatrix *m, QM *raw, QDP_Subset s) { SITES(s) m->d[i] = raw[i]; }
void QDP_extract_M(QM *raw, QDP_ColorMatrix *m, QDP_Subset s) { SITES(s) raw[i] = m->d[i]; }
void QDP_C_eq_c(QDP_Complex *r, C *c, QDP_Subset s) { SITES(s) r->d[i] = *c; }

/* ---------------------------------------------------------------- site helpers */
static inline C cmul(C a, C b) {
  C r;
  r.real = a.real * b.real - a.imag * b.imag;
  r.imag = a.real * b.imag + a.imag * b.real;
  return r;
}
static inline C cconjmul(C a, C b) {   /* conj(a) b */
  C r;
  r.real = a.real * b.real + a.imag * b.imag;
  r.imag = a.real * b.imag - a.imag * b.real;
  return r;
}
static inline void mv(QV *r, const QM *m, const QV *v) {   /* r = m v */
  QV t;
  for (int a = 0; a < 3; a++) {
    C s = {0, 0};
    for (int b = 0; b < 3; b++) {
      C p = cmul(m->e[a][b], v->c[b]);
      s.real += p.real;
      s.imag += p.imag;
    }
    t.c[a] = s;
  }
  *r = t;
}
static inline void mav(QV *r, const QM *m, const QV *v) {   /* r = m^+ v */
  QV t;
  for (int a = 0; a < 3; a++) {
    C s = {0, 0};
    for (int b = 0; b < 3; b++) {
      C p = cconjmul(m->e[b][a], v->c[b]);
      s.real += p.real;
      s.imag += p.imag;
    }
    t.c[a] = s;
  }
  *r = t;
}
/* r = op(a) op(b): ta / tb select the adjoint */
static inline void mm(QM *r, const QM *x, int ta, const QM *y, int tb) {
  QM t;
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) {
      C s = {0, 0};
      for (int k = 0; k < 3; k++) {
        C u = ta ? x->e[k][a] : x->e[a][k];
        C v = tb ? y->e[b][k] : y->e[k][b];
        if (ta) u.imag = -u.imag;
        if (tb) v.imag = -v.imag;
        C p = cmul(u, v);
        s.real += p.real;
        s.imag += p.imag;
      }
      t.e[a][b] = s;
    }
  *r = t;
}

/* ---------------------------------------------------------------- vectors */
void QDP_V_eq_zero(QDP_ColorVector *r, QDP_Subset s) { SITES(s) memset(&r->d[i], 0, sizeof(QV)); }
void QDP_V_eq_V(QDP_ColorVector *r, QDP_ColorVector *a, QDP_Subset s) { SITES(s) r->d[i] = a->d[i]; }

#define VLOOP(s, ...)                                    \
  SITES(s) for (int c = 0; c < 3; c++) {                 \
    C *rr = &r->d[i].c[c];                               \
    (void)rr;                                            \
    __VA_ARGS__;                                         \
  }
void QDP_V_peq_V(QDP_ColorVector *r, QDP_ColorVector *a, QDP_Subset s) {
  VLOOP(s, { rr->real += a->d[i].c[c].real; rr->imag += a->d[i].c[c].imag; })
}
void QDP_V_meq_V(QDP_ColorVector *r, QDP_ColorVector *a, QDP_Subset s) {
  VLOOP(s, { rr->real -= a->d[i].c[c].real; rr->imag -= a->d[i].c[c].imag; })
}
void QDP_V_eq_V_plus_V(QDP_ColorVector *r, QDP_ColorVector *a, QDP_ColorVector *b, QDP_Subset s) {
  VLOOP(s, {
    R x = a->d[i].c[c].real + b->d[i].c[c].real, y = a->d[i].c[c].imag + b->d[i].c[c].imag;
    rr->real = x; rr->imag = y;
  })
}
void QDP_V_eq_V_minus_V(QDP_ColorVector *r, QDP_ColorVector *a, QDP_ColorVector *b, QDP_Subset s) {
  VLOOP(s, {
    R x = a->d[i].c[c].real - b->d[i].c[c].real, y = a->d[i].c[c].imag - b->d[i].c[c].imag;
    rr->real = x; rr->imag = y;
  })
}
void QDP_V_eq_r_times_V(QDP_ColorVector *r, QLA_Real *f, QDP_ColorVector *a, QDP_Subset s) {
  const R k = *f;
  VLOOP(s, { rr->real = k * a->d[i].c[c].real; rr->imag = k * a->d[i].c[c].imag; })
}
void QDP_V_peq_r_times_V(QDP_ColorVector *r, QLA_Real *f, QDP_ColorVector *a, QDP_Subset s) {
  const R k = *f;
  VLOOP(s, { rr->real += k * a->d[i].c[c].real; rr->imag += k * a->d[i].c[c].imag; })
}
void QDP_V_meq_r_times_V(QDP_ColorVector *r, QLA_Real *f, QDP_ColorVector *a, QDP_Subset s) {
  const R k = *f;
  VLOOP(s, { rr->real -= k * a->d[i].c[c].real; rr->imag -= k * a->d[i].c[c].imag; })
}
void QDP_V_eq_r_times_V_plus_V(QDP_ColorVector *r, QLA_Real *f, QDP_ColorVector *a, QDP_ColorVector *b,
                               QDP_Subset s) {
  const R k = *f;
  VLOOP(s, {
    R x = k * a->d[i].c[c].real + b->d[i].c[c].real, y = k * a->d[i].c[c].imag + b->d[i].c[c].imag;
    rr->real = x; rr->imag = y;
  })
}
void QDP_V_eq_r_times_V_minus_V(QDP_ColorVector *r, QLA_Real *f, QDP_ColorVector *a, QDP_ColorVector *b,
                                QDP_Subset s) {
  const R k = *f;
  VLOOP(s, {
    R x = k * a->d[i].c[c].real - b->d[i].c[c].real, y = k * a->d[i].c[c].imag - b->d[i].c[c].imag;
    rr->real = x; rr->imag = y;
  })
}
void QDP_V_eq_c_times_V(QDP_ColorVector *r, QLA_Complex *z, QDP_ColorVector *a, QDP_Subset s) {
  const C k = *z;
  VLOOP(s, { *rr = cmul(k, a->d[i].c[c]); })
}
void QDP_V_peq_c_times_V(QDP_ColorVector *r, QLA_Complex *z, QDP_ColorVector *a, QDP_Subset s) {
  const C k = *z;
  VLOOP(s, { C p = cmul(k, a->d[i].c[c]); rr->real += p.real; rr->imag += p.imag; })
}
void QDP_V_meq_c_times_V(QDP_ColorVector *r, QLA_Complex *z, QDP_ColorVector *a, QDP_Subset s) {
  const C k = *z;
  VLOOP(s, { C p = cmul(k, a->d[i].c[c]); rr->real -= p.real; rr->imag -= p.imag; })
}
void QDP_V_eq_c_times_V_plus_V(QDP_ColorVector *r, QLA_Complex *z, QDP_ColorVector *a, QDP_ColorVector *b,
                               QDP_Subset s) {
  const C k = *z;
  VLOOP(s, {
    C p = cmul(k, a->d[i].c[c]);
    R x = p.real + b->d[i].c[c].real, y = p.imag + b->d[i].c[c].imag;
    rr->real = x; rr->imag = y;
  })
}

/* vectorised forms: n independent operations */
void QDP_V_veq_zero(QDP_ColorVector **r, QDP_Subset s, int n) { for (int k = 0; k < n; k++) QDP_V_eq_zero(r[k], s); }
void QDP_V_veq_V(QDP_ColorVector **r, QDP_ColorVector **a, QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) QDP_V_eq_V(r[k], a[k], s);
}
void QDP_V_vpeq_V(QDP_ColorVector **r, QDP_ColorVector **a, QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) QDP_V_peq_V(r[k], a[k], s);
}
void QDP_V_vmeq_V(QDP_ColorVector **r, QDP_ColorVector **a, QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) QDP_V_meq_V(r[k], a[k], s);
}
void QDP_V_veq_V_plus_V(QDP_ColorVector **r, QDP_ColorVector **a, QDP_ColorVector **b, QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) QDP_V_eq_V_plus_V(r[k], a[k], b[k], s);
}
void QDP_V_veq_V_minus_V(QDP_ColorVector **r, QDP_ColorVector **a, QDP_ColorVector **b, QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) QDP_V_eq_V_minus_V(r[k], a[k], b[k], s);
}
void QDP_V_veq_r_times_V(QDP_ColorVector **r, QLA_Real *f, QDP_ColorVector **a, QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) QDP_V_eq_r_times_V(r[k], &f[k], a[k], s);
}
void QDP_V_vpeq_r_times_V(QDP_ColorVector **r, QLA_Real *f, QDP_ColorVector **a, QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) QDP_V_peq_r_times_V(r[k], &f[k], a[k], s);
}
void QDP_V_vmeq_r_times_V(QDP_ColorVector **r, QLA_Real *f, QDP_ColorVector **a, QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) QDP_V_meq_r_times_V(r[k], &f[k], a[k], s);
}
void QDP_V_vpeq_c_times_V(QDP_ColorVector **r, QLA_Complex *z, QDP_ColorVector **a, QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) QDP_V_peq_c_times_V(r[k], &z[k], a[k], s);
}
void QDP_V_veq_r_times_V_plus_V(QDP_ColorVector **r, QLA_Real *f, QDP_ColorVector **a, QDP_ColorVector **b,
                                QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) QDP_V_eq_r_times_V_plus_V(r[k], &f[k], a[k], b[k], s);
}
void QDP_V_veq_c_times_V_plus_V(QDP_ColorVector **r, QLA_Complex *z, QDP_ColorVector **a, QDP_ColorVector **b,
                                QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) QDP_V_eq_c_times_V_plus_V(r[k], &z[k], a[k], b[k], s);
}

/* shifts: forward brings the value at x + shift to x, backward at x - shift */
void QDP_V_eq_sV(QDP_ColorVector *r, QDP_ColorVector *a, QDP_Shift sh, QDP_ShiftDir dir, QDP_Subset s) {
  const int *t = dir == QDP_forward ? sh->fwd : sh->bck;
  SITES(s) r->d[i] = a->d[t[i]];
}
void QDP_V_veq_sV(QDP_ColorVector **r, QDP_ColorVector **a, QDP_Shift *sh, QDP_ShiftDir *dir, QDP_Subset s,
                  int n) {
  for (int k = 0; k < n; k++) QDP_V_eq_sV(r[k], a[k], sh[k], dir[k], s);
}
void QDP_V_vpeq_M_times_V(QDP_ColorVector **r, QDP_ColorMatrix **m, QDP_ColorVector **a, QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) SITES(s) {
      QV t;
      mv(&t, &m[k]->d[i], &a[k]->d[i]);
      for (int c = 0; c < 3; c++) {
        r[k]->d[i].c[c].real += t.c[c].real;
        r[k]->d[i].c[c].imag += t.c[c].imag;
      }
    }
}
void QDP_V_veq_Ma_times_V(QDP_ColorVector **r, QDP_ColorMatrix **m, QDP_ColorVector **a, QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) SITES(s) mav(&r[k]->d[i], &m[k]->d[i], &a[k]->d[i]);
}

void QDP_V_eq_funcit(QDP_ColorVector *r, void (*f)(QV *, int), QDP_Subset s) { SITES(s) f(&r->d[i], i); }

/* reductions (double accumulation) */
void QDP_r_eq_norm2_V(QLA_Real *r, QDP_ColorVector *a, QDP_Subset s) {
  double acc = 0;
  SITES_SUM(s, acc) for (int c = 0; c < 3; c++) {
      const C z = a->d[i].c[c];
      acc += (double)z.real * z.real + (double)z.imag * z.imag;
    }
  *r = acc;
}
void QDP_r_veq_norm2_V(QLA_Real *r, QDP_ColorVector **a, QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) QDP_r_eq_norm2_V(&r[k], a[k], s);
}
void QDP_c_eq_V_dot_V(QLA_Complex *r, QDP_ColorVector *a, QDP_ColorVector *b, QDP_Subset s) {
  double re = 0, im = 0;
  SITES_SUM(s, re, im) for (int c = 0; c < 3; c++) {
      const C x = a->d[i].c[c], y = b->d[i].c[c];
      re += (double)x.real * y.real + (double)x.imag * y.imag;
      im += (double)x.real * y.imag - (double)x.imag * y.real;
    }
  r->real = re;
  r->imag = im;
}
void QDP_c_veq_V_dot_V(QLA_Complex *r, QDP_ColorVector **a, QDP_ColorVector **b, QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) QDP_c_eq_V_dot_V(&r[k], a[k], b[k], s);
}
void QDP_r_eq_re_V_dot_V(QLA_Real *r, QDP_ColorVector *a, QDP_ColorVector *b, QDP_Subset s) {
  QLA_Complex z;
  QDP_c_eq_V_dot_V(&z, a, b, s);
  *r = z.real;
}
void QDP_r_veq_re_V_dot_V(QLA_Real *r, QDP_ColorVector **a, QDP_ColorVector **b, QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) QDP_r_eq_re_V_dot_V(&r[k], a[k], b[k], s);
}

/* ---------------------------------------------------------------- matrices */
void QDP_M_eq_zero(QDP_ColorMatrix *r, QDP_Subset s) { SITES(s) memset(&r->d[i], 0, sizeof(QM)); }
void QDP_M_eq_M(QDP_ColorMatrix *r, QDP_ColorMatrix *a, QDP_Subset s) { SITES(s) r->d[i] = a->d[i]; }
void QDP_M_peq_M(QDP_ColorMatrix *r, QDP_ColorMatrix *a, QDP_Subset s) {
  SITES(s) for (int x = 0; x < 3; x++) for (int y = 0; y < 3; y++) {
        r->d[i].e[x][y].real += a->d[i].e[x][y].real;
        r->d[i].e[x][y].imag += a->d[i].e[x][y].imag;
      }
}
void QDP_M_eqm_Ma(QDP_ColorMatrix *r, QDP_ColorMatrix *a, QDP_Subset s) {
  SITES(s) {
    QM t;
    for (int x = 0; x < 3; x++)
      for (int y = 0; y < 3; y++) {
        t.e[x][y].real = -a->d[i].e[y][x].real;
        t.e[x][y].imag = a->d[i].e[y][x].imag;
      }
    r->d[i] = t;
  }
}
void QDP_M_eq_r_times_M(QDP_ColorMatrix *r, QLA_Real *f, QDP_ColorMatrix *a, QDP_Subset s) {
  const R k = *f;
  SITES(s) for (int x = 0; x < 3; x++) for (int y = 0; y < 3; y++) {
        r->d[i].e[x][y].real = k * a->d[i].e[x][y].real;
        r->d[i].e[x][y].imag = k * a->d[i].e[x][y].imag;
      }
}
void QDP_M_peq_r_times_M(QDP_ColorMatrix *r, QLA_Real *f, QDP_ColorMatrix *a, QDP_Subset s) {
  const R k = *f;
  SITES(s) for (int x = 0; x < 3; x++) for (int y = 0; y < 3; y++) {
        r->d[i].e[x][y].real += k * a->d[i].e[x][y].real;
        r->d[i].e[x][y].imag += k * a->d[i].e[x][y].imag;
      }
}
void QDP_M_eq_C_times_M(QDP_ColorMatrix *r, QDP_Complex *z, QDP_ColorMatrix *a, QDP_Subset s) {
  SITES(s) for (int x = 0; x < 3; x++) for (int y = 0; y < 3; y++) r->d[i].e[x][y] = cmul(z->d[i], a->d[i].e[x][y]);
}
void QDP_M_eq_M_times_M(QDP_ColorMatrix *r, QDP_ColorMatrix *a, QDP_ColorMatrix *b, QDP_Subset s) {
  SITES(s) mm(&r->d[i], &a->d[i], 0, &b->d[i], 0);
}
void QDP_M_eq_M_times_Ma(QDP_ColorMatrix *r, QDP_ColorMatrix *a, QDP_ColorMatrix *b, QDP_Subset s) {
  SITES(s) mm(&r->d[i], &a->d[i], 0, &b->d[i], 1);
}
void QDP_M_eq_Ma_times_M(QDP_ColorMatrix *r, QDP_ColorMatrix *a, QDP_ColorMatrix *b, QDP_Subset s) {
  SITES(s) mm(&r->d[i], &a->d[i], 1, &b->d[i], 0);
}
void QDP_M_eq_sM(QDP_ColorMatrix *r, QDP_ColorMatrix *a, QDP_Shift sh, QDP_ShiftDir dir, QDP_Subset s) {
  const int *t = dir == QDP_forward ? sh->fwd : sh->bck;
  SITES(s) r->d[i] = a->d[t[i]];
}
void QDP_M_eq_funct(QDP_ColorMatrix *r, void (*f)(QM *, int[]), QDP_Subset s) {
  SITES(s) {
    int x[4];
    memcpy(x, QDP_shim_coords[i], sizeof x);
    f(&r->d[i], x);
  }
}
void QDP_r_eq_norm2_M(QLA_Real *r, QDP_ColorMatrix *a, QDP_Subset s) {
  double acc = 0;
  SITES_SUM(s, acc) for (int x = 0; x < 3; x++) for (int y = 0; y < 3; y++) {
        const C z = a->d[i].e[x][y];
        acc += (double)z.real * z.real + (double)z.imag * z.imag;
      }
  *r = acc;
}
void QDP_m_eq_sum_M(QM *r, QDP_ColorMatrix *a, QDP_Subset s) {
  double re[3][3] = {{0}}, im[3][3] = {{0}};
  SITES_SERIAL(s) for (int x = 0; x < 3; x++) for (int y = 0; y < 3; y++) {
        re[x][y] += a->d[i].e[x][y].real;
        im[x][y] += a->d[i].e[x][y].imag;
      }
  for (int x = 0; x < 3; x++)
    for (int y = 0; y < 3; y++) {
      r->e[x][y].real = re[x][y];
      r->e[x][y].imag = im[x][y];
    }
}

/* ---------------------------------------------------------------- force algebra */
void QDP_M_eq_Ma(QDP_ColorMatrix *r, QDP_ColorMatrix *a, QDP_Subset s) {
  SITES(s) {
    QM t;
    for (int x = 0; x < 3; x++)
      for (int y = 0; y < 3; y++) {
        t.e[x][y].real = a->d[i].e[y][x].real;
        t.e[x][y].imag = -a->d[i].e[y][x].imag;
      }
    r->d[i] = t;
  }
}
void QDP_M_peq_Ma(QDP_ColorMatrix *r, QDP_ColorMatrix *a, QDP_Subset s) {
  SITES(s) {
    QM t;
    for (int x = 0; x < 3; x++)
      for (int y = 0; y < 3; y++) {
        t.e[x][y].real = r->d[i].e[x][y].real + a->d[i].e[y][x].real;
        t.e[x][y].imag = r->d[i].e[x][y].imag - a->d[i].e[y][x].imag;
      }
    r->d[i] = t;
  }
}
void QDP_M_eqm_M(QDP_ColorMatrix *r, QDP_ColorMatrix *a, QDP_Subset s) {
  SITES(s) for (int x = 0; x < 3; x++) for (int y = 0; y < 3; y++) {
        r->d[i].e[x][y].real = -a->d[i].e[x][y].real;
        r->d[i].e[x][y].imag = -a->d[i].e[x][y].imag;
      }
}
void QDP_M_meq_M(QDP_ColorMatrix *r, QDP_ColorMatrix *a, QDP_Subset s) {
  SITES(s) for (int x = 0; x < 3; x++) for (int y = 0; y < 3; y++) {
        r->d[i].e[x][y].real -= a->d[i].e[x][y].real;
        r->d[i].e[x][y].imag -= a->d[i].e[x][y].imag;
      }
}
/* traceless anti-Hermitian part: (a - a^+)/2 minus its trace / 3 on the diagonal */
void QDP_M_eq_antiherm_M(QDP_ColorMatrix *r, QDP_ColorMatrix *a, QDP_Subset s) {
  SITES(s) {
    const QM *m = &a->d[i];
    QM t;
    double trim = 0;
    for (int k = 0; k < 3; k++) trim += m->e[k][k].imag;
    for (int x = 0; x < 3; x++)
      for (int y = 0; y < 3; y++) {
        t.e[x][y].real = 0.5 * (m->e[x][y].real - m->e[y][x].real);
        t.e[x][y].imag = 0.5 * (m->e[x][y].imag + m->e[y][x].imag);
      }
    for (int k = 0; k < 3; k++) t.e[k][k].imag -= trim / 3.0;
    r->d[i] = t;
  }
}
void QDP_M_eq_r_times_M_plus_M(QDP_ColorMatrix *r, QLA_Real *f, QDP_ColorMatrix *a, QDP_ColorMatrix *b,
                               QDP_Subset s) {
  const R k = *f;
  SITES(s) for (int x = 0; x < 3; x++) for (int y = 0; y < 3; y++) {
        const R re = k * a->d[i].e[x][y].real + b->d[i].e[x][y].real;
        const R im = k * a->d[i].e[x][y].imag + b->d[i].e[x][y].imag;
        r->d[i].e[x][y].real = re;
        r->d[i].e[x][y].imag = im;
      }
}
void QDP_M_eq_Ma_times_Ma(QDP_ColorMatrix *r, QDP_ColorMatrix *a, QDP_ColorMatrix *b, QDP_Subset s) {
  SITES(s) mm(&r->d[i], &a->d[i], 1, &b->d[i], 1);
}
static inline void m_acc(QM *r, const QM *t, R sign) {
  for (int x = 0; x < 3; x++)
    for (int y = 0; y < 3; y++) {
      r->e[x][y].real += sign * t->e[x][y].real;
      r->e[x][y].imag += sign * t->e[x][y].imag;
    }
}
void QDP_M_peq_M_times_M(QDP_ColorMatrix *r, QDP_ColorMatrix *a, QDP_ColorMatrix *b, QDP_Subset s) {
  SITES(s) {
    QM t;
    mm(&t, &a->d[i], 0, &b->d[i], 0);
    m_acc(&r->d[i], &t, 1);
  }
}
void QDP_M_meq_M_times_M(QDP_ColorMatrix *r, QDP_ColorMatrix *a, QDP_ColorMatrix *b, QDP_Subset s) {
  SITES(s) {
    QM t;
    mm(&t, &a->d[i], 0, &b->d[i], 0);
    m_acc(&r->d[i], &t, -1);
  }
}
void QDP_M_peq_M_times_Ma(QDP_ColorMatrix *r, QDP_ColorMatrix *a, QDP_ColorMatrix *b, QDP_Subset s) {
  SITES(s) {
    QM t;
    mm(&t, &a->d[i], 0, &b->d[i], 1);
    m_acc(&r->d[i], &t, 1);
  }
}
/* outer product r_xy = v_x conj(w_y) */
void QDP_M_eq_V_times_Va(QDP_ColorMatrix *r, QDP_ColorVector *v, QDP_ColorVector *w, QDP_Subset s) {
  SITES(s) for (int x = 0; x < 3; x++) for (int y = 0; y < 3; y++) r->d[i].e[x][y] = cconjmul(w->d[i].c[y], v->d[i].c[x]);
}
void QDP_M_vpeq_V_times_Va(QDP_ColorMatrix **r, QDP_ColorVector **v, QDP_ColorVector **w, QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) SITES(s) for (int x = 0; x < 3; x++) for (int y = 0; y < 3; y++) {
          const C p = cconjmul(w[k]->d[i].c[y], v[k]->d[i].c[x]);
          r[k]->d[i].e[x][y].real += p.real;
          r[k]->d[i].e[x][y].imag += p.imag;
        }
}
void QDP_V_veq_M_times_V(QDP_ColorVector **r, QDP_ColorMatrix **m, QDP_ColorVector **v, QDP_Subset s, int n) {
  for (int k = 0; k < n; k++) SITES(s) mv(&r[k]->d[i], &m[k]->d[i], &v[k]->d[i]);
}
