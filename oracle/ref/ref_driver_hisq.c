/* ref_driver_hisq.c -- HISQ link construction through the reference's own
   QOP_D3_hisq_create_L_from_G (QOPQDP 0.21.1 lib/hisq_links_p.c, compiled
   unmodified against qdp_shim), with raw FP64 arrays in and out.  It reads
   the link sets out of the reference's QOP_D3_FermionLinksHisq, whose layout
   is internal to the reference (include/qop_d3_internal.h), so this unit is
   built like one of the reference's own D3 units.  Test infrastructure. */
#define QOP_Precision 'D'
#define QOP_Colors 3
#define QOP_Nc 3
#define QDP_Precision 'D'
#define QDP_Colors 3
#define QDP_Nc 3
#define QLA_Precision 'D'
#define QLA_Colors 3
#define QLA_Nc 3
#include <string.h>
#include <qop_internal.h>

static void m_to_raw(double *raw, QDP_D3_ColorMatrix *m, double f) {
  const double *d = (const double *)m->d;
  for (long i = 0; i < 18L * QDP_shim_V; i++) raw[i] = f * d[i];
}

/* hc: fat7 one_link, three_staple, five_staple, seven_staple, lepage;
   asqtad one_link, three_staple, five_staple, seven_staple, lepage, naik;
   difference one_link, naik (U(3) group, analytic projection).  Outputs,
   V x 18 doubles per direction: fat[4k + mu], lng[4k + mu] for the n_naiks
   link sets (unscaled, as QOP_asqtad_extract_L_to_qdp gives them), W[mu]
   the U(3)-projected links (may be NULL), dfat / dlng the Naik-epsilon
   derivative links (want_deps; may be NULL). */
int qr_hisq_links(const double hc[13], int n_naiks, const double *eps_naik, double *gauge[4], double *fat[],
                  double *lng[], double *W[4], double *dfat[4], double *dlng[4]) {
  QOP_info_t info = QOP_INFO_ZERO;
  QOP_opt_t opt[2] = {{"want_deps", dfat ? 1.0 : 0.0, NULL}, {"want_aux", 1.0, NULL}};
  QOP_hisq_links_set_opts(opt, 2);
  QOP_hisq_coeffs_t c;
  memset(&c, 0, sizeof c);
  c.n_naiks = n_naiks;
  for (int k = 0; k < n_naiks; k++) c.eps_naik[k] = eps_naik[k];
  c.ugroup = QOP_UNITARIZE_U3;
  c.umethod = QOP_UNITARIZE_ANALYTIC;
  c.fat7_one_link = hc[0];
  c.fat7_three_staple = hc[1];
  c.fat7_five_staple = hc[2];
  c.fat7_seven_staple = hc[3];
  c.fat7_lepage = hc[4];
  c.asqtad_one_link = hc[5];
  c.asqtad_three_staple = hc[6];
  c.asqtad_five_staple = hc[7];
  c.asqtad_seven_staple = hc[8];
  c.asqtad_lepage = hc[9];
  c.asqtad_naik = hc[10];
  c.difference_one_link = hc[11];
  c.difference_naik = hc[12];
  QDP_D3_ColorMatrix *g[4];
  for (int mu = 0; mu < 4; mu++) {
    g[mu] = QDP_D3_create_M();
    memcpy(g[mu]->d, gauge[mu], sizeof(double) * 18 * QDP_shim_V);
  }
  QOP_D3_GaugeField *gf = QOP_D3_create_G_from_qdp(g);
  QOP_D3_FermionLinksHisq *flh = QOP_D3_hisq_create_L_from_G(&info, &c, gf);
  /* the asqtad handles hold the links x 1/2 (lib/asqtad_dslash_p.c:195-200) */
  for (int k = 0; k < n_naiks; k++)
    for (int mu = 0; mu < 4; mu++) {
      m_to_raw(fat[4 * k + mu], flh->fn[k]->fatlinks[mu], 2.0);
      m_to_raw(lng[4 * k + mu], flh->fn[k]->longlinks[mu], 2.0);
    }
  if (W)
    for (int mu = 0; mu < 4; mu++) m_to_raw(W[mu], flh->W_unitlinks[mu], 1.0);
  if (dfat && flh->fn_deps)
    for (int mu = 0; mu < 4; mu++) {
      m_to_raw(dfat[mu], flh->fn_deps->fatlinks[mu], 2.0);
      m_to_raw(dlng[mu], flh->fn_deps->longlinks[mu], 2.0);
    }
  QOP_D3_hisq_destroy_L(flh);
  QOP_D3_destroy_G(gf);
  for (int mu = 0; mu < 4; mu++) QDP_D3_destroy_M(g[mu]);
  return info.status;
}

/* force[mu] (V x 18 doubles, accumulated into) += the HISQ fermion force of
   QOP_D3_hisq_force_multi_qdp (lib/hisq_force_p.c:44-58) for the links
   QOP_D3_hisq_create_L_from_G builds from `gauge` (coefficients as in
   qr_hisq_links, Naik epsilons eps_naik[n_naiks]), with the raw vectors
   x[k] (V x 6) weighted by res[k] and grouped by Naik term as n_orders[k]
   says; force_filter is the QOP_hisq_force_set_opts option (5e-5 by
   default in the reference) */
int qr_hisq_force(const double hc[13], int n_naiks, const double *eps_naik, double *gauge[4], double *force[4],
                  const double *res, double *x[], const int *n_orders, double force_filter) {
  QOP_info_t info = QOP_INFO_ZERO;
  QOP_opt_t fopt[1] = {{"force_filter", force_filter, NULL}};
  if (QOP_hisq_force_set_opts(fopt, 1) != QOP_SUCCESS) return QOP_FAIL;
  QOP_opt_t opt[2] = {{"want_deps", n_naiks > 1 ? 1.0 : 0.0, NULL}, {"want_aux", 1.0, NULL}};
  QOP_hisq_links_set_opts(opt, 2);
  QOP_hisq_coeffs_t c;
  memset(&c, 0, sizeof c);
  c.n_naiks = n_naiks;
  for (int k = 0; k < n_naiks; k++) c.eps_naik[k] = eps_naik[k];
  c.ugroup = QOP_UNITARIZE_U3;
  c.umethod = QOP_UNITARIZE_RATIONAL;   /* the force path of the analytic U(3) derivative (lib/hisq_force_fnmat_p.c:138-160) */
  c.fat7_one_link = hc[0];
  c.fat7_three_staple = hc[1];
  c.fat7_five_staple = hc[2];
  c.fat7_seven_staple = hc[3];
  c.fat7_lepage = hc[4];
  c.asqtad_one_link = hc[5];
  c.asqtad_three_staple = hc[6];
  c.asqtad_five_staple = hc[7];
  c.asqtad_seven_staple = hc[8];
  c.asqtad_lepage = hc[9];
  c.asqtad_naik = hc[10];
  c.difference_one_link = hc[11];
  c.difference_naik = hc[12];
  int nterms = 0;
  for (int k = 0; k < n_naiks; k++) nterms += n_orders[k];
  QDP_D3_ColorMatrix *g[4], *f[4];
  QDP_D3_ColorVector *xv[nterms];
  QLA_D_Real r[nterms];
  int no[n_naiks];
  for (int k = 0; k < n_naiks; k++) no[k] = n_orders[k];
  for (int mu = 0; mu < 4; mu++) {
    g[mu] = QDP_D3_create_M();
    f[mu] = QDP_D3_create_M();
    memcpy(g[mu]->d, gauge[mu], sizeof(double) * 18 * QDP_shim_V);
    memcpy(f[mu]->d, force[mu], sizeof(double) * 18 * QDP_shim_V);
  }
  for (int k = 0; k < nterms; k++) {
    xv[k] = QDP_D3_create_V();
    memcpy(xv[k]->d, x[k], sizeof(double) * 6 * QDP_shim_V);
    r[k] = res[k];
  }
  QOP_D3_GaugeField *gf = QOP_D3_create_G_from_qdp(g);
  QOP_D3_FermionLinksHisq *flh = QOP_D3_hisq_create_L_from_G(&info, &c, gf);
  QOP_D3_hisq_force_multi_qdp(&info, flh, f, &c, r, xv, no);
  for (int mu = 0; mu < 4; mu++) {
    memcpy(force[mu], f[mu]->d, sizeof(double) * 18 * QDP_shim_V);
    QDP_D3_destroy_M(g[mu]);
    QDP_D3_destroy_M(f[mu]);
  }
  for (int k = 0; k < nterms; k++) QDP_D3_destroy_V(xv[k]);
  QOP_D3_hisq_destroy_L(flh);
  QOP_D3_destroy_G(gf);
  return info.status;
}
