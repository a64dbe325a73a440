// fields.cu -- ColorVector / GaugeField handles and raw <-> device copies.
// Reference: lib/common_p.c:36-190 (create/extract/destroy from raw),
// include/qop_internal.h:125-141 (QOP_qdp_eq_raw: evenodd picks the half of
// a full-volume raw array), lib/common_p.c:455-526 (QOP_rephase_G).
#include "fields.cuh"
#include "reduce.cuh"
#include "dslash.cuh"

namespace qopb {

// raw AoS parity block (site, comp, re/im) -> SoA [comp][site] complex
template <typename TD, typename TS>
__global__ void k_raw_to_soa(c2<TD> *__restrict__ d, const TS *__restrict__ raw, int ncomp, i64 Vh) {
  i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (i >= Vh) return;
  for (int c = 0; c < ncomp; c++) {
    const TS *s = raw + (i * ncomp + c) * 2;
    d[c * Vh + i] = mk<TD>((TD)s[0], (TD)s[1]);
  }
}
template <typename TD, typename TS>
__global__ void k_soa_to_raw(TD *__restrict__ raw, const c2<TS> *__restrict__ s, int ncomp, i64 Vh, double scale) {
  i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (i >= Vh) return;
  for (int c = 0; c < ncomp; c++) {
    c2<TS> v = s[c * Vh + i];
    raw[(i * ncomp + c) * 2] = (TD)(scale * (double)v.x);
    raw[(i * ncomp + c) * 2 + 1] = (TD)(scale * (double)v.y);
  }
}

template <typename TD, typename TS>
void raw_to_dev(c2<TD> *dfield, const TS *raw, int ncomp, int eo) {
  Context &c = ctx();
  const Geom &g = c.g;
  for (int p = 0; p < 2; p++) {
    if (eo != QOP_EVENODD && eo != p) continue;
    size_t n = (size_t)g.Vh * ncomp * 2;
    TS *stage = dalloc<TS>((i64)n);
    QCHECK(cudaMemcpyAsync(stage, raw + (size_t)p * n, n * sizeof(TS), cudaMemcpyHostToDevice, c.s));
    k_raw_to_soa<TD, TS><<<grid_for(g.Vh, 256), 256, 0, c.s>>>(dfield + (i64)p * ncomp * g.Vh, stage, ncomp, g.Vh);
    QLAUNCH();
    dfree(stage);
  }
  sync();
}

template <typename TD, typename TS>
void dev_to_raw(TD *raw, const c2<TS> *dfield, int ncomp, int eo, double scale) {
  Context &c = ctx();
  const Geom &g = c.g;
  for (int p = 0; p < 2; p++) {
    if (eo != QOP_EVENODD && eo != p) continue;
    size_t n = (size_t)g.Vh * ncomp * 2;
    TD *stage = dalloc<TD>((i64)n);
    k_soa_to_raw<TD, TS><<<grid_for(g.Vh, 256), 256, 0, c.s>>>(stage, dfield + (i64)p * ncomp * g.Vh, ncomp, g.Vh, scale);
    QLAUNCH();
    QCHECK(cudaMemcpyAsync(raw + (size_t)p * n, stage, n * sizeof(TD), cudaMemcpyDeviceToHost, c.s));
    dfree(stage);
  }
  sync();
}

template void raw_to_dev<float, float>(c2<float> *, const float *, int, int);
template void raw_to_dev<double, double>(c2<double> *, const double *, int, int);
template void raw_to_dev<double, float>(c2<double> *, const float *, int, int);
template void dev_to_raw<float, float>(float *, const c2<float> *, int, int, double);
template void dev_to_raw<double, double>(double *, const c2<double> *, int, int, double);
template void dev_to_raw<float, double>(float *, const c2<double> *, int, int, double);

// ---------------------------------------------------------------- rephase
// common_p.c:455-526: boundary phase on the last slice (origin r0) and the
// staggered sign (-1)^{sum_j mask_j x_j} using unshifted coordinates
template <typename T>
__global__ void k_rephase_G(c2<T> *m, Geom g, int bc_dir, int org, double phr, double phi, int bits) {
  i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (s >= 2 * g.Vh) return;
  int p = (int)(s / g.Vh), i = (int)(s % g.Vh);
  int x[4];
  site_coords(g, i, p, x);
  for (int j = 0; j < 4; j++) x[j] += g.O[j];   // global coordinates
  double fr = 1, fi = 0;
  if (bc_dir >= 0) {
    int n = g.GL[bc_dir];
    int rshift = (x[bc_dir] + n - org) % n;
    if (rshift == n - 1) { fr = phr; fi = phi; }
  }
  if (bits) {
    int t = 0;
    for (int j = 0; j < 4; j++) t += ((bits >> j) & 1) * x[j];
    if (t & 1) { fr = -fr; fi = -fi; }
  }
  if (fr == 1 && fi == 0) return;
  c2<T> *b = m + (i64)p * 9 * g.Vh + i;
  for (int e = 0; e < 9; e++) {
    c2<T> v = b[e * g.Vh];
    b[e * g.Vh] = mk<T>((T)(fr * v.x - fi * v.y), (T)(fr * v.y + fi * v.x));
  }
}

template <typename T>
void rephase_gauge(GaugeT<T> *G, const int *r0, const QOP_Complex *bc, const int *sign) {
  const Geom &g = ctx().g;
  for (int i = 0; i < 4; i++) {
    int bc_dir = -1;
    double pr = 1, pi = 0;
    if (bc && (bc[i].re != 1. || bc[i].im != 0.)) { bc_dir = i; pr = bc[i].re; pi = bc[i].im; }
    int bits = sign ? sign[i] : 0;
    int org = (bc_dir >= 0 && r0) ? r0[i] : 0;
    k_rephase_G<T><<<grid_for(2 * g.Vh, 256), 256, 0, ctx().s>>>(G->d + (i64)i * 18 * g.Vh, g, bc_dir, org, pr, pi, bits);
    QLAUNCH();
  }
}
template void rephase_gauge<float>(GaugeT<float> *, const int *, const QOP_Complex *, const int *);
template void rephase_gauge<double>(GaugeT<double> *, const int *, const QOP_Complex *, const int *);

template <typename T>
GaugeT<T> *gauge_new() {
  const Geom &g = ctx().g;
  GaugeT<T> *G = new GaugeT<T>();
  G->d = dalloc<c2<T>>(4 * 18 * g.Vh);
  dzero(G->d, sizeof(c2<T>) * 4 * 18 * g.Vh);
  handle_register(G);
  return G;
}
template <typename T>
void gauge_destroy(GaugeT<T> *G) {
  if (!G) return;
  dfree(G->d);
  delete[] G->r0; delete[] G->bc; delete[] G->signmask;
  handle_forget(G);
  delete G;
}
template GaugeT<float> *gauge_new<float>();
template GaugeT<double> *gauge_new<double>();
template void gauge_destroy<float>(GaugeT<float> *);
template void gauge_destroy<double>(GaugeT<double> *);

template <typename T>
VecT<T> *vec_new() {
  const Geom &g = ctx().g;
  VecT<T> *v = new VecT<T>();
  v->d = dalloc<c2<T>>(vec_elems(g));
  dzero(v->d, sizeof(c2<T>) * vec_elems(g));
  handle_register(v);
  return v;
}
template <typename T>
void vec_destroy(VecT<T> *v) {
  if (!v) return;
  dfree(v->d);
  handle_forget(v);
  delete v;
}
template VecT<float> *vec_new<float>();
template VecT<double> *vec_new<double>();
template void vec_destroy<float>(VecT<float> *);
template void vec_destroy<double>(VecT<double> *);

}  // namespace qopb
