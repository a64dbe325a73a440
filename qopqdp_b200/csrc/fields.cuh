// fields.cuh -- handle constructors and raw copies (fields.cu, links.cu).
#pragma once
#include "qopb.h"

namespace qopb {

// raw full-volume AoS array (ncomp complex per site) <-> device SoA field
// [2][ncomp][Vh]; only the parity halves selected by eo are touched
template <typename TD, typename TS> void raw_to_dev(c2<TD> *dfield, const TS *raw, int ncomp, int eo);
template <typename TD, typename TS> void dev_to_raw(TD *raw, const c2<TS> *dfield, int ncomp, int eo, double scale);

template <typename T> VecT<T> *vec_new();
template <typename T> void vec_destroy(VecT<T> *v);
template <typename T> GaugeT<T> *gauge_new();
template <typename T> void gauge_destroy(GaugeT<T> *G);
template <typename T> void rephase_gauge(GaugeT<T> *G, const int *r0, const QOP_Complex *bc, const int *sign);

// links.cu
template <typename T> FlaT<T> *fla_alloc(int nlinks);
template <typename T> void fla_load_fwd(FlaT<T> *f, const c2<T> *fat, const c2<T> *lng, double scale);
template <typename T> void fla_extract_fwd(FlaT<T> *f, c2<T> *fat, c2<T> *lng, double scale);
template <typename T> void fla_rephase(FlaT<T> *f, const int *r0, const QOP_Complex *bc, const int *sign);
template <typename T> FlaT<T> *fla_from_G(QOP_info_t *info, const QOP_asqtad_coeffs_t *coef, GaugeT<T> *gfat,
                                          GaugeT<T> *glong);
template <typename T> HisqT<T> *hisq_from_G(QOP_info_t *info, const QOP_hisq_coeffs_t *coef, GaugeT<T> *gauge);
template <typename T> void hisq_destroy(HisqT<T> *h);
template <typename T> FlaT<T> *fla_scaled_copy(FlaT<T> *src, double s);
template <typename T> void fla_peq(FlaT<T> *f, FlaT<T> *g);
void sloppy_invalidate(void *fla_any);   // drop reduced-precision copies (mixed.cu)

// force.cu: F_mu += -2 TA(U_mu deriv_mu^+) for the sources x (eps weights)
template <typename T>
void asqtad_force(QOP_info_t *info, GaugeT<T> *G, GaugeT<T> *F, const QOP_asqtad_coeffs_t *cf, const double *eps,
                  VecT<T> *const *x, int nsrc);
// force.cu: HISQ force (F_mu += TA(U_mu (2 deriv_mu)^+)) from the handle's
// auxiliary U, V, W fields; sources grouped by Naik epsilon (n_orders)
template <typename T>
void hisq_force(QOP_info_t *info, HisqT<T> *h, GaugeT<T> *F, const QOP_hisq_coeffs_t *cf, const double *res,
                VecT<T> *const *x, const int *n_orders);

}  // namespace qopb
