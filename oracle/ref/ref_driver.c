/* ref_driver.c -- plain C entry points into the reference's own asqtad path
   (QOPQDP 0.21.1 lib/asqtad_dslash_p.c, lib/asqtad_invert_p.c,
   lib/invert_cg_p.c, compiled unmodified against qdp_shim) for the test
   suite: raw FP64 arrays in QOP raw site order in, raw FP64 arrays out.
   prec 0 runs the reference's F3 (single precision) build of the path,
   prec 1 its D3 build.  Test infrastructure only. */
#include <stdlib.h>
#include <string.h>
#include "qop_qdp.h"

static int g_L[4];

int qr_init(const int latsize[4]) {
  QOP_layout_t lay = QOP_LAYOUT_ZERO;
  memcpy(g_L, latsize, sizeof g_L);
  lay.latdim = 4;
  lay.latsize = g_L;
  lay.machdim = -1;
  return QOP_init(&lay);
}

int qr_finalize(void) { return QOP_finalize(); }

int qr_verbose(int level) { return QOP_verbose(level); }

int qr_set_opt(const char *tag, double value) {
  QOP_opt_t o;
  o.tag = (char *)tag;
  o.value = value;
  o.extra = NULL;
  return QOP_asqtad_invert_set_opts(&o, 1);
}

/* ------------------------------------------------------------- fields */
static QDP_F3_ColorVector *vf_from(const double *raw) {
  QDP_F3_ColorVector *v = QDP_F3_create_V();
  if (raw) {
    float *d = (float *)v->d;
    for (long i = 0; i < 6L * QDP_shim_V; i++) d[i] = (float)raw[i];
  }
  return v;
}
static QDP_D3_ColorVector *vd_from(const double *raw) {
  QDP_D3_ColorVector *v = QDP_D3_create_V();
  if (raw) memcpy(v->d, raw, sizeof(double) * 6 * QDP_shim_V);
  return v;
}
static void vf_to(double *raw, QDP_F3_ColorVector *v) {
  const float *d = (const float *)v->d;
  for (long i = 0; i < 6L * QDP_shim_V; i++) raw[i] = d[i];
}
static void vd_to(double *raw, QDP_D3_ColorVector *v) { memcpy(raw, v->d, sizeof(double) * 6 * QDP_shim_V); }

/* links: fat[mu], lng[mu] are V x 18 doubles (lng may be NULL: no Naik) */
void *qr_fla_create(int prec, double *const fat[4], double *const lng[4]) {
  const long n = 18L * QDP_shim_V;
  if (prec == 0) {
    QDP_F3_ColorMatrix *fl[4], *ll[4];
    for (int mu = 0; mu < 4; mu++) {
      fl[mu] = QDP_F3_create_M();
      for (long i = 0; i < n; i++) ((float *)fl[mu]->d)[i] = (float)fat[mu][i];
      if (lng) {
        ll[mu] = QDP_F3_create_M();
        for (long i = 0; i < n; i++) ((float *)ll[mu]->d)[i] = (float)lng[mu][i];
      }
    }
    void *r = QOP_F3_asqtad_create_L_from_qdp(fl, lng ? ll : NULL);
    for (int mu = 0; mu < 4; mu++) {
      QDP_F3_destroy_M(fl[mu]);
      if (lng) QDP_F3_destroy_M(ll[mu]);
    }
    return r;
  }
  QDP_D3_ColorMatrix *fl[4], *ll[4];
  for (int mu = 0; mu < 4; mu++) {
    fl[mu] = QDP_D3_create_M();
    memcpy(fl[mu]->d, fat[mu], sizeof(double) * n);
    if (lng) {
      ll[mu] = QDP_D3_create_M();
      memcpy(ll[mu]->d, lng[mu], sizeof(double) * n);
    }
  }
  void *r = QOP_D3_asqtad_create_L_from_qdp(fl, lng ? ll : NULL);
  for (int mu = 0; mu < 4; mu++) {
    QDP_D3_destroy_M(fl[mu]);
    if (lng) QDP_D3_destroy_M(ll[mu]);
  }
  return r;
}

void qr_fla_destroy(int prec, void *fla) {
  if (prec == 0)
    QOP_F3_asqtad_destroy_L((QOP_F3_FermionLinksAsqtad *)fla);
  else
    QOP_D3_asqtad_destroy_L((QOP_D3_FermionLinksAsqtad *)fla);
}

/* out (V x 6, full volume) is read and written: sites outside eo_out keep
   their values, as the reference's field does */
int qr_dslash(int prec, void *fla, double mass, double *out, const double *in, int eo_out, int eo_in) {
  QOP_info_t info = QOP_INFO_ZERO;
  if (prec == 0) {
    QDP_F3_ColorVector *o = vf_from(out), *i = vf_from(in);
    QOP_F3_asqtad_dslash_qdp(&info, (QOP_F3_FermionLinksAsqtad *)fla, (float)mass, o, i, eo_out, eo_in);
    vf_to(out, o);
    QDP_F3_destroy_V(o);
    QDP_F3_destroy_V(i);
  } else {
    QDP_D3_ColorVector *o = vd_from(out), *i = vd_from(in);
    QOP_D3_asqtad_dslash_qdp(&info, (QOP_D3_FermionLinksAsqtad *)fla, mass, o, i, eo_out, eo_in);
    vd_to(out, o);
    QDP_D3_destroy_V(o);
    QDP_D3_destroy_V(i);
  }
  return info.status;
}

/* out holds the initial guess on entry and the solution on return */
int qr_invert(int prec, void *fla, QOP_invert_arg_t *ia, QOP_resid_arg_t *ra, double mass, double *out,
              const double *in, double *flops) {
  QOP_info_t info = QOP_INFO_ZERO;
  if (prec == 0) {
    QDP_F3_ColorVector *o = vf_from(out), *i = vf_from(in);
    QOP_F3_asqtad_invert_qdp(&info, (QOP_F3_FermionLinksAsqtad *)fla, ia, ra, (float)mass, o, i);
    vf_to(out, o);
    QDP_F3_destroy_V(o);
    QDP_F3_destroy_V(i);
  } else {
    QDP_D3_ColorVector *o = vd_from(out), *i = vd_from(in);
    QOP_D3_asqtad_invert_qdp(&info, (QOP_D3_FermionLinksAsqtad *)fla, ia, ra, mass, o, i);
    vd_to(out, o);
    QDP_D3_destroy_V(o);
    QDP_D3_destroy_V(i);
  }
  if (flops) *flops = info.final_flop;
  return info.status;
}

/* nsrc sources in[s], each with nmass[s] masses masses[s][k]; out[s][k]
   are zero-initialised by the caller and receive the solutions */
int qr_invert_multi(int prec, void *fla, QOP_invert_arg_t *ia, QOP_resid_arg_t **ra[], double *masses[],
                    int nmass[], double **out[], double *in[], int nsrc, double *flops) {
  QOP_info_t info = QOP_INFO_ZERO;
  if (prec == 0) {
    QDP_F3_ColorVector *iv[nsrc], **ov[nsrc];
    float *mv[nsrc];
    for (int s = 0; s < nsrc; s++) {
      iv[s] = vf_from(in[s]);
      ov[s] = (QDP_F3_ColorVector **)malloc(sizeof(void *) * nmass[s]);
      mv[s] = (float *)malloc(sizeof(float) * nmass[s]);
      for (int k = 0; k < nmass[s]; k++) {
        ov[s][k] = vf_from(out[s][k]);
        mv[s][k] = (float)masses[s][k];
      }
    }
    QOP_F3_asqtad_invert_multi_qdp(&info, (QOP_F3_FermionLinksAsqtad *)fla, ia, ra, mv, nmass, ov, iv, nsrc);
    for (int s = 0; s < nsrc; s++) {
      for (int k = 0; k < nmass[s]; k++) {
        vf_to(out[s][k], ov[s][k]);
        QDP_F3_destroy_V(ov[s][k]);
      }
      QDP_F3_destroy_V(iv[s]);
      free(ov[s]);
      free(mv[s]);
    }
  } else {
    QDP_D3_ColorVector *iv[nsrc], **ov[nsrc];
    for (int s = 0; s < nsrc; s++) {
      iv[s] = vd_from(in[s]);
      ov[s] = (QDP_D3_ColorVector **)malloc(sizeof(void *) * nmass[s]);
      for (int k = 0; k < nmass[s]; k++) ov[s][k] = vd_from(out[s][k]);
    }
    QOP_D3_asqtad_invert_multi_qdp(&info, (QOP_D3_FermionLinksAsqtad *)fla, ia, ra, masses, nmass, ov, iv, nsrc);
    for (int s = 0; s < nsrc; s++) {
      for (int k = 0; k < nmass[s]; k++) {
        vd_to(out[s][k], ov[s][k]);
        QDP_D3_destroy_V(ov[s][k]);
      }
      QDP_D3_destroy_V(iv[s]);
      free(ov[s]);
    }
  }
  if (flops) *flops = info.final_flop;
  return info.status;
}

/* eigCG (QOP_asqtad_invert_set_opts "cg" = 1) is not part of this build:
   its Lanczos stage needs the reference's linear-algebra files.  The
   solvers reach these only with that option set. */
QOP_status_t QOP_F3_invert_eigcg_V(void *linop, void *ia, void *ra, void *out, void *in, void *p, void *sub,
                                   void *eigcg) {
  QDP_abort(1);
  return QOP_FAIL;
}
QOP_status_t QOP_D3_invert_eigcg_V(void *linop, void *ia, void *ra, void *out, void *in, void *p, void *sub,
                                   void *eigcg) {
  QDP_abort(1);
  return QOP_FAIL;
}

/* ------------------------------------------------------------- links */
/* QOP_D3_rephase_G_qdp (lib/common_p.c:529-543) on raw links (V x 18 doubles
   per direction, changed in place); bc = 4 complex phases as 8 doubles */
int qr_rephase_G(double *links[4], const int r0[4], const double bc[8], const int signmask[4]) {
  QDP_D3_ColorMatrix *g[4];
  QOP_Complex ph[4];
  int r[4], sm[4];
  for (int mu = 0; mu < 4; mu++) {
    g[mu] = QDP_D3_create_M();
    memcpy(g[mu]->d, links[mu], sizeof(double) * 18 * QDP_shim_V);
    ph[mu].re = bc[2 * mu];
    ph[mu].im = bc[2 * mu + 1];
    r[mu] = r0[mu];
    sm[mu] = signmask[mu];
  }
  QOP_bc_t b = {ph};
  QOP_staggered_sign_t s = {sm};
  QOP_D3_rephase_G_qdp(g, r, &b, &s);
  for (int mu = 0; mu < 4; mu++) {
    memcpy(links[mu], g[mu]->d, sizeof(double) * 18 * QDP_shim_V);
    QDP_D3_destroy_M(g[mu]);
  }
  return 0;
}

/* asqtad fat and long links from a gauge field through the reference's
   QOP_D3_asqtad_create_L_from_G (lib/asqtad_dslash_p.c:642-665; the
   smearing of make_imp_links) and QOP_D3_asqtad_extract_L_to_qdp; coeffs
   = one_link, three_staple, five_staple, seven_staple, lepage, naik */
int qr_asqtad_links_from_G(const double coeffs[6], double *gauge[4], double *fat[4], double *lng[4]) {
  QOP_info_t info = QOP_INFO_ZERO;
  QDP_D3_ColorMatrix *g[4], *fl[4], *ll[4];
  for (int mu = 0; mu < 4; mu++) {
    g[mu] = QDP_D3_create_M();
    memcpy(g[mu]->d, gauge[mu], sizeof(double) * 18 * QDP_shim_V);
    fl[mu] = QDP_D3_create_M();
    ll[mu] = QDP_D3_create_M();
  }
  QOP_asqtad_coeffs_t c;
  c.one_link = coeffs[0];
  c.three_staple = coeffs[1];
  c.five_staple = coeffs[2];
  c.seven_staple = coeffs[3];
  c.lepage = coeffs[4];
  c.naik = coeffs[5];
  QOP_D3_GaugeField *gf = QOP_D3_create_G_from_qdp(g);
  QOP_D3_FermionLinksAsqtad *fla = QOP_D3_asqtad_create_L_from_G(&info, &c, gf);
  QOP_D3_asqtad_extract_L_to_qdp(fl, lng ? ll : NULL, fla);
  for (int mu = 0; mu < 4; mu++) {
    memcpy(fat[mu], fl[mu]->d, sizeof(double) * 18 * QDP_shim_V);
    if (lng) memcpy(lng[mu], ll[mu]->d, sizeof(double) * 18 * QDP_shim_V);
    QDP_D3_destroy_M(g[mu]);
    QDP_D3_destroy_M(fl[mu]);
    QDP_D3_destroy_M(ll[mu]);
  }
  QOP_D3_asqtad_destroy_L(fla);
  QOP_D3_destroy_G(gf);
  return info.status;
}

/* host threads for the OpenMP site loops (QDP's threading); returns the
   number in effect */
#ifdef _OPENMP
#include <omp.h>
#endif
int qr_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

/* ------------------------------------------------------------- forces */
/* force[mu] (V x 18 doubles, accumulated into) += the asqtad fermion force
   of QOP_D3_asqtad_force_multi_qdp (lib/asqtad_force_p.c:15-38) for the
   gauge field `gauge`, coefficients as in qr_asqtad_links_from_G, and nsrc
   raw vectors x[k] (V x 6) with weights eps[k]; fnmat_src_min (the
   QOP_asqtad_force_set_opts option) selects the ASVEC algorithm for
   nsrc < fnmat_src_min, else FNMAT */
int qr_asqtad_force(const double coeffs[6], double *gauge[4], double *force[4], const double *eps, double *x[],
                    int nsrc, int fnmat_src_min) {
  QOP_info_t info = QOP_INFO_ZERO;
  QOP_opt_t o[1] = {{"fnmat_src_min", (double)fnmat_src_min, NULL}};
  if (QOP_asqtad_force_set_opts(o, 1) != QOP_SUCCESS) return QOP_FAIL;
  QDP_D3_ColorMatrix *g[4], *f[4];
  QDP_D3_ColorVector *xv[nsrc];
  double e[nsrc];
  for (int mu = 0; mu < 4; mu++) {
    g[mu] = QDP_D3_create_M();
    f[mu] = QDP_D3_create_M();
    memcpy(g[mu]->d, gauge[mu], sizeof(double) * 18 * QDP_shim_V);
    memcpy(f[mu]->d, force[mu], sizeof(double) * 18 * QDP_shim_V);
  }
  for (int k = 0; k < nsrc; k++) {
    xv[k] = vd_from(x[k]);
    e[k] = eps[k];
  }
  QOP_asqtad_coeffs_t c;
  c.one_link = coeffs[0];
  c.three_staple = coeffs[1];
  c.five_staple = coeffs[2];
  c.seven_staple = coeffs[3];
  c.lepage = coeffs[4];
  c.naik = coeffs[5];
  QOP_D3_asqtad_force_multi_qdp(&info, g, f, &c, e, xv, nsrc);
  for (int mu = 0; mu < 4; mu++) {
    memcpy(force[mu], f[mu]->d, sizeof(double) * 18 * QDP_shim_V);
    QDP_D3_destroy_M(g[mu]);
    QDP_D3_destroy_M(f[mu]);
  }
  for (int k = 0; k < nsrc; k++) QDP_D3_destroy_V(xv[k]);
  return info.status;
}

/* deriv[mu] (V x 18 doubles, accumulated into) += the derivative of
   Re sum tr[midF^+ fat + midN^+ long] with respect to the gauge links, as
   the reference's QOP_D3_asqtad_deriv forms it (lib/asqtad_force_fnmat_p.c;
   midN may be NULL) */
int qr_asqtad_deriv(const double coeffs[6], double *gauge[4], double *deriv[4], double *midF[4], double *midN[4]) {
  QOP_info_t info = QOP_INFO_ZERO;
  QDP_D3_ColorMatrix *g[4], *d[4], *mf[4], *mn[4];
  for (int mu = 0; mu < 4; mu++) {
    g[mu] = QDP_D3_create_M();
    d[mu] = QDP_D3_create_M();
    mf[mu] = QDP_D3_create_M();
    mn[mu] = QDP_D3_create_M();
    memcpy(g[mu]->d, gauge[mu], sizeof(double) * 18 * QDP_shim_V);
    memcpy(d[mu]->d, deriv[mu], sizeof(double) * 18 * QDP_shim_V);
    memcpy(mf[mu]->d, midF[mu], sizeof(double) * 18 * QDP_shim_V);
    if (midN) memcpy(mn[mu]->d, midN[mu], sizeof(double) * 18 * QDP_shim_V);
  }
  QOP_asqtad_coeffs_t c;
  c.one_link = coeffs[0];
  c.three_staple = coeffs[1];
  c.five_staple = coeffs[2];
  c.seven_staple = coeffs[3];
  c.lepage = coeffs[4];
  c.naik = coeffs[5];
  QOP_D3_asqtad_deriv(&info, g, d, &c, mf, midN ? mn : NULL);
  for (int mu = 0; mu < 4; mu++) {
    memcpy(deriv[mu], d[mu]->d, sizeof(double) * 18 * QDP_shim_V);
    QDP_D3_destroy_M(g[mu]);
    QDP_D3_destroy_M(d[mu]);
    QDP_D3_destroy_M(mf[mu]);
    QDP_D3_destroy_M(mn[mu]);
  }
  return info.status;
}
