// api.cu -- the exported QOP_F3_* / QOP_D3_* C ABI (include/qop.h).
// One template per entry point, instantiated for F3 (float) and D3
// (double).  Handles are the internal objects behind opaque pointers.
// Every entry point catches internal failures and reports them in
// info->status (or a NULL handle); nothing calls exit().
// Reference signatures: include/qop_pc.h:50-115 (fields), :219-306
// (asqtad links, dslash), :316-371 (inverters), :471-483 (HISQ).
#include "qopb.h"
#include "fields.cuh"
#include "solvers.cuh"
#include <vector>

using namespace qopb;

namespace {

template <typename T> struct Hd;
template <> struct Hd<float> {
  typedef QOP_F3_ColorVector V; typedef QOP_F3_GaugeField G;
  typedef QOP_F3_FermionLinksAsqtad L; typedef QOP_F3_FermionLinksHisq H;
};
template <> struct Hd<double> {
  typedef QOP_D3_ColorVector V; typedef QOP_D3_GaugeField G;
  typedef QOP_D3_FermionLinksAsqtad L; typedef QOP_D3_FermionLinksHisq H;
};
template <typename T> VecT<T> *iv(typename Hd<T>::V *h) { return reinterpret_cast<VecT<T> *>(h); }
template <typename T> GaugeT<T> *ig(typename Hd<T>::G *h) { return reinterpret_cast<GaugeT<T> *>(h); }
template <typename T> FlaT<T> *il(typename Hd<T>::L *h) { return reinterpret_cast<FlaT<T> *>(h); }
template <typename T> HisqT<T> *ih(typename Hd<T>::H *h) { return reinterpret_cast<HisqT<T> *>(h); }

void report(QOP_info_t *info, const Fail &e, const char *fn) {
  fprintf(stderr, "%s: %s\n", fn, e.msg.c_str());
  if (info) info->status = e.status;
}
#define TRY try {
#define CATCH(info, ret) } catch (Fail &e) { report(info, e, __func__); return ret; }
#define CATCHV(info) } catch (Fail &e) { report(info, e, __func__); return; }

template <typename T> void need_handle(const void *h, const char *what) { handle_check(h, what); }

// ---------------------------------------------------------------- fields
template <typename T, typename R> VecT<T> *create_V(const R *src, int eo) {
  require_init("create_V_from_raw");
  VecT<T> *v = vec_new<T>();
  if (src) raw_to_dev<T, R>(v->d, src, 3, eo);
  else sync();
  return v;
}
template <typename T, typename R> void extract_V(R *dest, VecT<T> *v, int eo) {
  require_init("extract_V_to_raw");
  need_handle<T>(v, "ColorVector");
  dev_to_raw<R, T>(dest, v->d, 3, eo, 1.0);
}
template <typename T, typename R> GaugeT<T> *create_G(R *links[], int eo) {
  require_init("create_G_from_raw");
  GaugeT<T> *G = gauge_new<T>();
  const Geom &g = ctx().g;
  for (int mu = 0; mu < 4; mu++) raw_to_dev<T, R>(G->d + (i64)mu * 18 * g.Vh, links[mu], 9, eo);
  return G;
}
template <typename T, typename R> void extract_G(R *dest[], GaugeT<T> *G, int eo) {
  require_init("extract_G_to_raw");
  need_handle<T>(G, "GaugeField");
  const Geom &g = ctx().g;
  for (int mu = 0; mu < 4; mu++) dev_to_raw<R, T>(dest[mu], G->d + (i64)mu * 18 * g.Vh, 9, eo, 1.0);
}
template <typename T> void rephase_G(GaugeT<T> *G, int *r0, QOP_bc_t *bc, QOP_staggered_sign_t *sign) {
  require_init("rephase_G");
  need_handle<T>(G, "GaugeField");
  if (!r0 || !bc || !bc->phase || !sign || !sign->signmask) fail(QOP_FAIL, "rephase_G: NULL r0/bc/sign");
  // common_p.c:510-526 keeps a copy of the phases in the handle
  delete[] G->r0; delete[] G->bc; delete[] G->signmask;
  G->r0 = new int[4]; G->bc = new QOP_Complex[4]; G->signmask = new int[4];
  memcpy(G->r0, r0, 4 * sizeof(int));
  memcpy(G->bc, bc->phase, 4 * sizeof(QOP_Complex));
  memcpy(G->signmask, sign->signmask, 4 * sizeof(int));
  rephase_gauge<T>(G, r0, bc->phase, sign->signmask);
  sync();
}

// ---------------------------------------------------------------- links
template <typename T, typename R> FlaT<T> *create_L_raw(R *fat[], R *lng[], int eo) {
  require_init("asqtad_create_L_from_raw");
  const Geom &g = ctx().g;
  const i64 F4 = 72 * g.Vh;
  c2<T> *df = dalloc<c2<T>>(F4), *dl = lng ? dalloc<c2<T>>(F4) : nullptr;
  dzero(df, sizeof(c2<T>) * F4);
  if (dl) dzero(dl, sizeof(c2<T>) * F4);
  for (int mu = 0; mu < 4; mu++) {
    raw_to_dev<T, R>(df + (i64)mu * 18 * g.Vh, fat[mu], 9, eo);
    if (dl) raw_to_dev<T, R>(dl + (i64)mu * 18 * g.Vh, lng[mu], 9, eo);
  }
  FlaT<T> *f = fla_alloc<T>(lng ? 16 : 8);
  fla_load_fwd<T>(f, df, dl, 0.5);
  dfree(df); if (dl) dfree(dl);
  sync();
  return f;
}
template <typename T, typename R> void load_L_raw(FlaT<T> *f, R *fat[], R *lng[], int eo) {
  require_init("asqtad_load_L_from_raw");
  need_handle<T>(f, "FermionLinksAsqtad");
  if ((lng != nullptr) != (f->nlinks == 16)) fail(QOP_FAIL, "load_L_from_raw: Naik links do not match the handle");
  const Geom &g = ctx().g;
  const i64 F4 = 72 * g.Vh;
  c2<T> *df = dalloc<c2<T>>(F4), *dl = lng ? dalloc<c2<T>>(F4) : nullptr;
  fla_extract_fwd<T>(f, df, dl, 2.0);   // keep the untouched parity
  for (int mu = 0; mu < 4; mu++) {
    raw_to_dev<T, R>(df + (i64)mu * 18 * g.Vh, fat[mu], 9, eo);
    if (dl) raw_to_dev<T, R>(dl + (i64)mu * 18 * g.Vh, lng[mu], 9, eo);
  }
  fla_load_fwd<T>(f, df, dl, 0.5);
  sloppy_invalidate((void *)f);
  if (f->shadow32) { fla_destroy((FlaT<float> *)f->shadow32); f->shadow32 = nullptr; }
  dfree(df); if (dl) dfree(dl);
  sync();
}
template <typename T, typename R> void extract_L_raw(R *fat[], R *lng[], FlaT<T> *f, int eo) {
  require_init("asqtad_extract_L_to_raw");
  need_handle<T>(f, "FermionLinksAsqtad");
  const Geom &g = ctx().g;
  const i64 F4 = 72 * g.Vh;
  c2<T> *df = dalloc<c2<T>>(F4), *dl = (f->nlinks == 16) ? dalloc<c2<T>>(F4) : nullptr;
  fla_extract_fwd<T>(f, df, dl, 2.0);
  for (int mu = 0; mu < 4; mu++) {
    dev_to_raw<R, T>(fat[mu], df + (i64)mu * 18 * g.Vh, 9, eo, 1.0);
    if (lng && dl) dev_to_raw<R, T>(lng[mu], dl + (i64)mu * 18 * g.Vh, 9, eo, 1.0);
  }
  dfree(df); if (dl) dfree(dl);
  sync();
}

// ---------------------------------------------------------------- operators
template <typename T> void dslash(QOP_info_t *info, FlaT<T> *f, double mass, VecT<T> *out, VecT<T> *in, int eo_out,
                                  int eo_in) {
  require_init("asqtad_dslash");
  need_handle<T>(f, "FermionLinksAsqtad");
  need_handle<T>(out, "ColorVector");
  need_handle<T>(in, "ColorVector");
  double t0 = wtime();
  Dslash<T>::apply(f, mass, out->d, in->d, eo_out, eo_in);
  sync();
  if (info) {
    info->final_sec = wtime() - t0;
    int nsub = (eo_out == QOP_EVENODD ? 2 : 1);
    info->final_flop = (eo_in != eo_out || eo_out == QOP_EVENODD) ? 0.5 * (2 * 8 * 9 * f->nlinks - 6) * nsub * ctx().g.Vh : 0;
    info->status = QOP_SUCCESS;
  }
}
template <typename T> void dslash_dir(QOP_info_t *info, FlaT<T> *f, int dir, int fb, double wtfat, double wtlong,
                                      VecT<T> *out, VecT<T> *in, int eo_out) {
  require_init("asqtad_dslash_dir");
  need_handle<T>(f, "FermionLinksAsqtad");
  if (dir < 0 || dir > 3) fail(QOP_FAIL, "dslash_dir: bad direction %d", dir);
  Dslash<T>::dslash_dir(f, dir, fb, wtfat, wtlong, out->d, in->d, eo_out);
  sync();
  if (info) info->status = QOP_SUCCESS;
}
template <typename T> void diaginv(QOP_info_t *info, double mass, VecT<T> *out, VecT<T> *in, int eo) {
  require_init("asqtad_diaginv");
  Blas<T>::scale(out->d, (double)((T)1.0 / (T)mass), in->d, vrange(ctx().g, eo));
  sync();
  if (info) info->status = QOP_SUCCESS;
}
template <typename T> double ddagd(QOP_info_t *info, FlaT<T> *f, double mass, VecT<T> *out, VecT<T> *in, int eo,
                                   bool norm) {
  require_init("asqtad_ddagd");
  need_handle<T>(f, "FermionLinksAsqtad");
  if (eo == QOP_EVENODD) fail(QOP_FAIL, "ddagd: eo must be QOP_EVEN or QOP_ODD");
  c2<T> *tmp = dalloc<c2<T>>(vec_elems(ctx().g));
  double r = Dslash<T>::ddagd(f, mass, out->d, in->d, eo, tmp, norm);
  dfree(tmp);
  sync();
  if (info) info->status = QOP_SUCCESS;
  return r;
}
template <typename T> void invert_api(QOP_info_t *info, FlaT<T> *f, QOP_invert_arg_t *ia, QOP_resid_arg_t *ra,
                                      double mass, VecT<T> *out, VecT<T> *in) {
  require_init("asqtad_invert");
  need_handle<T>(f, "FermionLinksAsqtad");
  need_handle<T>(out, "ColorVector");
  need_handle<T>(in, "ColorVector");
  if (!ia || !ra) fail(QOP_FAIL, "invert: NULL argument structs");
  invert<T>(info, f, ia, ra, mass, out->d, in->d);
}
template <typename T, typename R> void invert_multi_api(QOP_info_t *info, FlaT<T> *f, QOP_invert_arg_t *ia,
                                                        QOP_resid_arg_t **ra[], R *masses[], int nmass[],
                                                        typename Hd<T>::V **out_pt[], typename Hd<T>::V *in_pt[],
                                                        int nsrc) {
  require_init("asqtad_invert_multi");
  need_handle<T>(f, "FermionLinksAsqtad");
  if (nsrc < 1) fail(QOP_FAIL, "invert_multi: nsrc < 1");
  std::vector<std::vector<c2<T> *>> o(nsrc);
  std::vector<c2<T> **> op(nsrc);
  std::vector<c2<T> *> in(nsrc);
  std::vector<std::vector<double>> m(nsrc);
  std::vector<double *> mp(nsrc);
  for (int i = 0; i < nsrc; i++) {
    need_handle<T>(in_pt[i], "ColorVector");
    in[i] = iv<T>(in_pt[i])->d;
    for (int j = 0; j < nmass[i]; j++) {
      need_handle<T>(out_pt[i][j], "ColorVector");
      o[i].push_back(iv<T>(out_pt[i][j])->d);
      m[i].push_back((double)masses[i][j]);
    }
    op[i] = o[i].data();
    mp[i] = m[i].data();
  }
  invert_multi<T>(info, f, ia, ra, mp.data(), nmass, op.data(), in.data(), nsrc);
}

}  // namespace

#define QOPB_DEFINE_PC(PC, T, REAL)                                                                                 \
  extern "C" QOP_##PC##_ColorVector *QOP_##PC##_create_V_from_raw(REAL *src, QOP_evenodd_t eo) {                  \
    TRY return reinterpret_cast<QOP_##PC##_ColorVector *>(create_V<T, REAL>(src, eo)); CATCH(nullptr, nullptr)     \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_extract_V_to_raw(REAL *dest, QOP_##PC##_ColorVector *src, QOP_evenodd_t eo) {        \
    TRY extract_V<T, REAL>(dest, iv<T>(src), eo); CATCHV(nullptr)                                                   \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_destroy_V(QOP_##PC##_ColorVector *v) { TRY vec_destroy<T>(iv<T>(v)); CATCHV(nullptr) } \
  extern "C" QOP_##PC##_GaugeField *QOP_##PC##_create_G_from_raw(REAL *links[], QOP_evenodd_t eo) {               \
    TRY return reinterpret_cast<QOP_##PC##_GaugeField *>(create_G<T, REAL>(links, eo)); CATCH(nullptr, nullptr)    \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_extract_G_to_raw(REAL *dest[], QOP_##PC##_GaugeField *src, QOP_evenodd_t eo) {       \
    TRY extract_G<T, REAL>(dest, ig<T>(src), eo); CATCHV(nullptr)                                                   \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_destroy_G(QOP_##PC##_GaugeField *G) { TRY gauge_destroy<T>(ig<T>(G)); CATCHV(nullptr) } \
  extern "C" void QOP_##PC##_rephase_G(QOP_##PC##_GaugeField *G, int *r0, QOP_bc_t *bc, QOP_staggered_sign_t *s) { \
    TRY rephase_G<T>(ig<T>(G), r0, bc, s); CATCHV(nullptr)                                                          \
  }                                                                                                                 \
  extern "C" QOP_##PC##_FermionLinksAsqtad *QOP_##PC##_asqtad_create_L_from_raw(REAL *fat[], REAL *lng[],         \
                                                                                QOP_evenodd_t eo) {               \
    TRY return reinterpret_cast<QOP_##PC##_FermionLinksAsqtad *>(create_L_raw<T, REAL>(fat, lng, eo));             \
    CATCH(nullptr, nullptr)                                                                                         \
  }                                                                                                                 \
  extern "C" QOP_##PC##_FermionLinksAsqtad *QOP_##PC##_asqtad_create_L_from_G(                                     \
      QOP_info_t *info, QOP_asqtad_coeffs_t *coeffs, QOP_##PC##_GaugeField *gauge) {                               \
    TRY require_init(__func__); need_handle<T>(gauge, "GaugeField");                                               \
    return reinterpret_cast<QOP_##PC##_FermionLinksAsqtad *>(fla_from_G<T>(info, coeffs, ig<T>(gauge), nullptr));  \
    CATCH(info, nullptr)                                                                                            \
  }                                                                                                                 \
  extern "C" QOP_##PC##_FermionLinksAsqtad *QOP_##PC##_asqtad_create_L_from_G2(                                    \
      QOP_info_t *info, QOP_asqtad_coeffs_t *coeffs, QOP_##PC##_GaugeField *gFat, QOP_##PC##_GaugeField *gLong) {   \
    TRY require_init(__func__); need_handle<T>(gFat, "GaugeField"); need_handle<T>(gLong, "GaugeField");           \
    return reinterpret_cast<QOP_##PC##_FermionLinksAsqtad *>(fla_from_G<T>(info, coeffs, ig<T>(gFat), ig<T>(gLong))); \
    CATCH(info, nullptr)                                                                                            \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_asqtad_load_L_from_raw(QOP_##PC##_FermionLinksAsqtad *fla, REAL *fat[], REAL *lng[], \
                                                    QOP_evenodd_t eo) {                                           \
    TRY load_L_raw<T, REAL>(il<T>(fla), fat, lng, eo); CATCHV(nullptr)                                              \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_asqtad_extract_L_to_raw(REAL *fat[], REAL *lng[], QOP_##PC##_FermionLinksAsqtad *fla, \
                                                     QOP_evenodd_t eo) {                                          \
    TRY extract_L_raw<T, REAL>(fat, lng, il<T>(fla), eo); CATCHV(nullptr)                                           \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_asqtad_destroy_L(QOP_##PC##_FermionLinksAsqtad *fla) {                               \
    TRY FlaT<T> *f = il<T>(fla); if (!f) return;                                                                    \
    if (f->shadow32) fla_destroy((FlaT<float> *)f->shadow32);                                                       \
    fla_destroy<T>(f); CATCHV(nullptr)                                                                              \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_asqtad_rephase_L(QOP_##PC##_FermionLinksAsqtad *fla, int *r0, QOP_bc_t *bc,          \
                                              QOP_staggered_sign_t *sign) {                                       \
    TRY require_init(__func__); FlaT<T> *f = il<T>(fla); need_handle<T>(f, "FermionLinksAsqtad");                  \
    fla_rephase<T>(f, r0, bc ? bc->phase : nullptr, sign ? sign->signmask : nullptr);                               \
    sloppy_invalidate((void *)f);                                                                                   \
    if (f->shadow32) { fla_destroy((FlaT<float> *)f->shadow32); f->shadow32 = nullptr; }                            \
    sync(); CATCHV(nullptr)                                                                                         \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_asqtad_dslash(QOP_info_t *info, QOP_##PC##_FermionLinksAsqtad *fla, REAL mass,       \
                                           QOP_##PC##_ColorVector *out, QOP_##PC##_ColorVector *in,               \
                                           QOP_evenodd_t eo_out, QOP_evenodd_t eo_in) {                           \
    TRY dslash<T>(info, il<T>(fla), mass, iv<T>(out), iv<T>(in), eo_out, eo_in); CATCHV(info)                      \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_asqtad_dslash_dir(QOP_info_t *info, QOP_##PC##_FermionLinksAsqtad *fla, int dir,     \
                                               int fb, double wtfat, double wtlong, QOP_##PC##_ColorVector *out,  \
                                               QOP_##PC##_ColorVector *in, QOP_evenodd_t eo_out) {                \
    TRY dslash_dir<T>(info, il<T>(fla), dir, fb, wtfat, wtlong, iv<T>(out), iv<T>(in), eo_out); CATCHV(info)       \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_asqtad_diaginv(QOP_info_t *info, QOP_##PC##_FermionLinksAsqtad *fla, REAL mass,      \
                                            QOP_##PC##_ColorVector *out, QOP_##PC##_ColorVector *in,              \
                                            QOP_evenodd_t eo) {                                                   \
    (void)fla; TRY diaginv<T>(info, mass, iv<T>(out), iv<T>(in), eo); CATCHV(info)                                  \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_asqtad_ddagd(QOP_info_t *info, QOP_##PC##_FermionLinksAsqtad *fla, REAL mass,        \
                                          QOP_##PC##_ColorVector *out, QOP_##PC##_ColorVector *in,                \
                                          QOP_evenodd_t eo) {                                                     \
    TRY ddagd<T>(info, il<T>(fla), mass, iv<T>(out), iv<T>(in), eo, false); CATCHV(info)                           \
  }                                                                                                                 \
  extern "C" REAL QOP_##PC##_asqtad_ddagd_norm2(QOP_info_t *info, QOP_##PC##_FermionLinksAsqtad *fla, REAL mass,  \
                                                QOP_##PC##_ColorVector *out, QOP_##PC##_ColorVector *in,          \
                                                QOP_evenodd_t eo) {                                               \
    TRY return (REAL)ddagd<T>(info, il<T>(fla), mass, iv<T>(out), iv<T>(in), eo, true); CATCH(info, (REAL)-1)      \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_asqtad_invert(QOP_info_t *info, QOP_##PC##_FermionLinksAsqtad *fla,                  \
                                           QOP_invert_arg_t *ia, QOP_resid_arg_t *ra, REAL mass,                  \
                                           QOP_##PC##_ColorVector *out, QOP_##PC##_ColorVector *in) {             \
    TRY invert_api<T>(info, il<T>(fla), ia, ra, mass, iv<T>(out), iv<T>(in)); CATCHV(info)                         \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_asqtad_invert_multi(QOP_info_t *info, QOP_##PC##_FermionLinksAsqtad *fla,            \
                                                 QOP_invert_arg_t *ia, QOP_resid_arg_t **ra[], REAL *masses[],    \
                                                 int nmass[], QOP_##PC##_ColorVector **out[],                     \
                                                 QOP_##PC##_ColorVector *in[], int nsrc) {                        \
    TRY invert_multi_api<T, REAL>(info, il<T>(fla), ia, ra, masses, nmass, out, in, nsrc); CATCHV(info)            \
  }                                                                                                                 \
  extern "C" QOP_##PC##_FermionLinksHisq *QOP_##PC##_hisq_create_L_from_G(QOP_info_t *info,                      \
                                                                          QOP_hisq_coeffs_t *coeffs,              \
                                                                          QOP_##PC##_GaugeField *gauge) {         \
    TRY require_init(__func__); need_handle<T>(gauge, "GaugeField");                                               \
    return reinterpret_cast<QOP_##PC##_FermionLinksHisq *>(hisq_from_G<T>(info, coeffs, ig<T>(gauge)));            \
    CATCH(info, nullptr)                                                                                            \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_hisq_destroy_L(QOP_##PC##_FermionLinksHisq *h) {                                     \
    TRY hisq_destroy<T>(ih<T>(h)); CATCHV(nullptr)                                                                  \
  }                                                                                                                 \
  extern "C" QOP_##PC##_FermionLinksAsqtad **QOP_##PC##_get_asqtad_links_from_hisq(QOP_##PC##_FermionLinksHisq *h) { \
    return h ? reinterpret_cast<QOP_##PC##_FermionLinksAsqtad **>(ih<T>(h)->fn) : nullptr;                         \
  }                                                                                                                 \
  extern "C" QOP_##PC##_FermionLinksAsqtad *QOP_##PC##_get_asqtad_deps_links_from_hisq(                          \
      QOP_##PC##_FermionLinksHisq *h) {                                                                             \
    return h ? reinterpret_cast<QOP_##PC##_FermionLinksAsqtad *>(ih<T>(h)->fn_deps) : nullptr;                     \
  }

QOPB_DEFINE_PC(F3, float, float)
QOPB_DEFINE_PC(D3, double, double)

extern "C" QOP_F3_FermionLinksAsqtad *QOP_FD3_asqtad_create_L_from_L(QOP_D3_FermionLinksAsqtad *src) {
  TRY require_init(__func__); need_handle<double>(src, "FermionLinksAsqtad");
  FlaT<float> *f = fla_convert<float, double>(il<double>(src));
  sync();
  return reinterpret_cast<QOP_F3_FermionLinksAsqtad *>(f);
  CATCH(nullptr, nullptr)
}

// ---------------------------------------------------------------- fermion force
// Force fields share the gauge-field layout ([4 mu][2][9][Vh]); the force
// accumulates into the handle as in the reference (asqtad_force_fnmat_p.c:536-538).
namespace {
template <typename T, typename R>
void force_multi(QOP_info_t *info, GaugeT<T> *G, GaugeT<T> *F, QOP_asqtad_coeffs_t *coef, const R *eps,
                 VecT<T> *const *in, int nsrc) {
  require_init("asqtad_force");
  dd_refuse("asqtad_force");
  need_handle<T>(G, "GaugeField");
  need_handle<T>(F, "Force");
  if (!coef || !eps || !in || nsrc < 1) fail(QOP_FAIL, "asqtad_force: NULL coefficients / eps / sources or nsrc < 1");
  std::vector<double> e(nsrc);
  for (int i = 0; i < nsrc; i++) {
    need_handle<T>(in[i], "ColorVector");
    e[i] = (double)eps[i];
  }
  asqtad_force<T>(info, G, F, coef, e.data(), in, nsrc);
}
template <typename T, typename R>
void hisq_force_multi(QOP_info_t *info, HisqT<T> *h, GaugeT<T> *F, QOP_hisq_coeffs_t *coef, const R *eps,
                      VecT<T> *const *in, const int *n_orders) {
  require_init("hisq_force_multi");
  dd_refuse("hisq_force_multi");
  need_handle<T>(h, "FermionLinksHisq");
  need_handle<T>(F, "Force");
  if (!coef || !eps || !in || !n_orders) fail(QOP_FAIL, "hisq_force_multi: NULL coefficients / eps / sources / orders");
  if (coef->n_naiks < 1 || coef->n_naiks > QOP_MAX_NAIK || coef->n_naiks != h->n_naiks)
    fail(QOP_FAIL, "hisq_force_multi: n_naiks %d does not match the links (%d)", coef->n_naiks, h->n_naiks);
  int nterms = 0;
  for (int k = 0; k < coef->n_naiks; k++) {
    if (n_orders[k] < 0) fail(QOP_FAIL, "hisq_force_multi: negative n_orders_naik");
    nterms += n_orders[k];
  }
  if (nterms < 1) fail(QOP_FAIL, "hisq_force_multi: no sources");
  std::vector<double> e(nterms);
  for (int i = 0; i < nterms; i++) {
    need_handle<T>(in[i], "ColorVector");
    e[i] = (double)eps[i];
  }
  hisq_force<T>(info, h, F, coef, e.data(), in, n_orders);
}
}  // namespace

#define QOPB_DEFINE_FORCE(PC, T, REAL)                                                                            \
  extern "C" QOP_##PC##_Force *QOP_##PC##_create_F_from_raw(REAL *force[], QOP_evenodd_t eo) {                     \
    TRY return reinterpret_cast<QOP_##PC##_Force *>(create_G<T, REAL>(force, eo)); CATCH(nullptr, nullptr)          \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_extract_F_to_raw(REAL *dest[], QOP_##PC##_Force *src, QOP_evenodd_t eo) {            \
    TRY extract_G<T, REAL>(dest, reinterpret_cast<GaugeT<T> *>(src), eo); CATCHV(nullptr)                          \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_destroy_F(QOP_##PC##_Force *F) {                                                     \
    TRY gauge_destroy<T>(reinterpret_cast<GaugeT<T> *>(F)); CATCHV(nullptr)                                         \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_asqtad_force_multi(QOP_info_t *info, QOP_##PC##_GaugeField *gauge,                   \
                                                QOP_##PC##_Force *force, QOP_asqtad_coeffs_t *coef, REAL eps[],   \
                                                QOP_##PC##_ColorVector *in_pt[], int nsrc) {                      \
    TRY force_multi<T, REAL>(info, ig<T>(gauge), reinterpret_cast<GaugeT<T> *>(force), coef, eps,                  \
                             reinterpret_cast<VecT<T> *const *>(in_pt), nsrc);                                     \
    CATCHV(info)                                                                                                    \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_hisq_force_multi(QOP_info_t *info, QOP_##PC##_FermionLinksHisq *flh,                \
                                              QOP_##PC##_Force *force, QOP_hisq_coeffs_t *coef, REAL eps[],       \
                                              QOP_##PC##_ColorVector *in_pt[], int *n_orders_naik) {              \
    TRY hisq_force_multi<T, REAL>(info, ih<T>(flh), reinterpret_cast<GaugeT<T> *>(force), coef, eps,             \
                                  reinterpret_cast<VecT<T> *const *>(in_pt), n_orders_naik);                       \
    CATCHV(info)                                                                                                    \
  }                                                                                                                 \
  extern "C" void QOP_##PC##_asqtad_force(QOP_info_t *info, QOP_##PC##_GaugeField *gauge, QOP_##PC##_Force *force, \
                                          QOP_asqtad_coeffs_t *coef, REAL eps, QOP_##PC##_ColorVector *in_pt) {   \
    QOP_##PC##_asqtad_force_multi(info, gauge, force, coef, &eps, &in_pt, 1);                                      \
  }

QOPB_DEFINE_FORCE(F3, float, float)
QOPB_DEFINE_FORCE(D3, double, double)

// eigCG space introspection (no counterpart in the reference)
#define QOPB_DEFINE_EIGCG(PC, T)                                                                                   \
  extern "C" int QOPB_##PC##_eigcg_values(QOP_##PC##_FermionLinksAsqtad *L, QOP_evenodd_t eo, double *l, int max) { \
    TRY require_init("eigcg_values");                                                                              \
    need_handle<T>(L, "FermionLinksAsqtad");                                                                       \
    if (eo != QOP_EVEN && eo != QOP_ODD) fail(QOP_FAIL, "eigcg_values: eo must be QOP_EVEN or QOP_ODD");           \
    if (max > 0 && !l) fail(QOP_FAIL, "eigcg_values: NULL output");                                                \
    return eigcg_values<T>(reinterpret_cast<FlaT<T> *>(L), eo, l, max);                                            \
    CATCH(nullptr, -1)                                                                                             \
  }
QOPB_DEFINE_EIGCG(F3, float)
QOPB_DEFINE_EIGCG(D3, double)

// lib/asqtad_force.c:19-41: fnmat_src_min selects the normalisation of the
// reference's ASVEC algorithm for calls with fewer sources (asqtad_force in
// force.cu); veclength (ASVEC's block of sources) is validated and kept
// lib/hisq_force.c:29-52 (the reference has one HISQ force algorithm; its
// fnmat_src_min and veclength are validated and kept, force_filter is used
// by the U(3) projection's adjoint in force.cu)
extern "C" QOP_status_t QOP_hisq_force_set_opts(QOP_opt_t opts[], int nopts) {
  Options &o = ctx().opt;
  int fsm = o.hisq_fnmat_src_min, vl = o.hisq_veclength;
  double ff = o.hisq_force_filter;
  for (int i = 0; i < nopts; i++) {
    if (!opts[i].tag) continue;
    if (!strcmp(opts[i].tag, "fnmat_src_min")) fsm = (int)opts[i].value;
    else if (!strcmp(opts[i].tag, "veclength")) vl = (int)opts[i].value;
    else if (!strcmp(opts[i].tag, "force_filter")) ff = opts[i].value;
  }
  if (fsm < 0 || vl <= 0 || !(ff >= 0)) return QOP_FAIL;
  o.hisq_fnmat_src_min = fsm;
  o.hisq_veclength = vl;
  o.hisq_force_filter = ff;
  return QOP_SUCCESS;
}

extern "C" QOP_status_t QOP_asqtad_force_set_opts(QOP_opt_t opts[], int nopts) {
  int fsm = ctx().opt.force_fnmat_src_min, vl = ctx().opt.force_veclength;
  for (int i = 0; i < nopts; i++) {
    if (!opts[i].tag) continue;
    if (!strcmp(opts[i].tag, "fnmat_src_min")) fsm = (int)opts[i].value;
    else if (!strcmp(opts[i].tag, "veclength")) vl = (int)opts[i].value;
  }
  if (fsm < 0 || vl <= 0) return QOP_FAIL;
  ctx().opt.force_fnmat_src_min = fsm;
  ctx().opt.force_veclength = vl;
  return QOP_SUCCESS;
}
