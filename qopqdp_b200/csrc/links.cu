// links.cu -- FermionLinksAsqtad / FermionLinksHisq on the device.
// Reference: lib/asqtad_dslash_p.c:152-223 (convert_L: links x 1/2),
// :79-133 (double_store: bck(x) = -fwd(x - shift)^+), :391-455 and :458-633
// (compute_gen_staple / make_imp_links), :915-938 (extract_L: x 2),
// :1447-1482 (rephase_L), lib/hisq_links_p.c:62-256 (HISQ chain),
// lib/hisq_reunit_utilities_p.c:99-297 (U(3) projection).
// Link smearing and projection always run in FP64 on the device; the result
// is rounded once to the handle's precision.
#include "fields.cuh"
#include "reduce.cuh"
#include "dslash.cuh"
#include "mat3.cuh"
#include <cmath>

namespace qopb {


// ---------------------------------------------------------------- staples
// upper(x) = U_nu(x) [link(x+nu) U_nu(x+mu)^+]
// lower(x) = [U_nu(y)^+ link(y)] U_nu(y+mu),  y = x - nu
// SAVE: save = upper + lower, fl += coef save; else fl += coef upper; fl += coef lower
template <bool SAVE>
__global__ void k_staple(double2 *fl, double2 *save, const double2 *link, const double2 *Unu, int mu, int nu,
                         double coef, Geom g) {
  i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (s >= 2 * g.Vh) return;
  const int p = (int)(s / g.Vh), i = (int)(s % g.Vh);
  const i64 Vh = g.Vh;
  int x[4], y[4];
  site_coords(g, i, p, x);
  int pn, in_, pm, im, py, iy, pym, iym;
  shifted(g, x, nu, 1, y); par_idx(g, y, pn, in_);
  shifted(g, x, mu, 1, y); par_idx(g, y, pm, im);
  int yy[4];
  shifted(g, x, nu, -1, yy); par_idx(g, yy, py, iy);
  shifted(g, yy, mu, 1, y); par_idx(g, y, pym, iym);
  M3 t1 = mul_na(ld3(fptr(link, g, pn, in_), Vh), ld3(fptr(Unu, g, pm, im), Vh));
  M3 up = mul(ld3(fptr(Unu, g, p, i), Vh), t1);
  t1 = mul_an(ld3(fptr(Unu, g, py, iy), Vh), ld3(fptr(link, g, py, iy), Vh));
  M3 lo = mul(t1, ld3(fptr(Unu, g, pym, iym), Vh));
  double2 *F = fl + (i64)p * 9 * Vh + i;
  if (SAVE) {
    double2 *S = save + (i64)p * 9 * Vh + i;
#pragma unroll
    for (int e = 0; e < 9; e++) {
      double2 v = make_double2(up.e[e].x + lo.e[e].x, up.e[e].y + lo.e[e].y);
      S[e * Vh] = v;
      double2 f = F[e * Vh];
      F[e * Vh] = make_double2(f.x + coef * v.x, f.y + coef * v.y);
    }
  } else {
#pragma unroll
    for (int e = 0; e < 9; e++) {
      double2 f = F[e * Vh];
      f.x += coef * up.e[e].x; f.y += coef * up.e[e].y;
      f.x += coef * lo.e[e].x; f.y += coef * lo.e[e].y;
      F[e * Vh] = f;
    }
  }
}

__global__ void k_scale_field(double2 *d, const double2 *s, double c, i64 n) {
  i64 k = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (k >= n) return;
  double2 v = s[k];
  d[k] = make_double2(c * v.x, c * v.y);
}

// ll(x) = naik U(x) [U(x+mu) U(x+2mu)]
__global__ void k_naik(double2 *ll, const double2 *U, int mu, double naik, Geom g) {
  i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (s >= 2 * g.Vh) return;
  const int p = (int)(s / g.Vh), i = (int)(s % g.Vh);
  int x[4], y[4], p1, i1, p2, i2;
  site_coords(g, i, p, x);
  shifted(g, x, mu, 1, y); par_idx(g, y, p1, i1);
  shifted(g, x, mu, 2, y); par_idx(g, y, p2, i2);
  M3 t = mul(ld3(fptr(U, g, p1, i1), g.Vh), ld3(fptr(U, g, p2, i2), g.Vh));
  M3 r = mul(ld3(fptr(U, g, p, i), g.Vh), t);
#pragma unroll
  for (int e = 0; e < 9; e++) { r.e[e].x *= naik; r.e[e].y *= naik; }
  st3(ll + (i64)p * 9 * g.Vh + i, g.Vh, r);
}

static void staple(double2 *fl, double2 *save, const double2 *link, const double2 *Unu, int mu, int nu, double coef) {
  const Geom &g = ctx().g;
  int grid = grid_for(2 * g.Vh, 128);
  if (save) k_staple<true><<<grid, 128, 0, ctx().s>>>(fl, save, link, Unu, mu, nu, coef, g);
  else k_staple<false><<<grid, 128, 0, ctx().s>>>(fl, nullptr, link, Unu, mu, nu, coef, g);
  QLAUNCH();
}

// make_imp_links (asqtad_dslash_p.c:458-633): gf, gfLong, fl, ll are
// [4][2][9][Vh] FP64 fields; ll may be null (no Naik term)
static double make_imp_links(const QOP_asqtad_coeffs_t *cf, const double2 *gf, const double2 *gfLong, double2 *fl,
                             double2 *ll) {
  const Geom &g = ctx().g;
  const i64 F = 18 * g.Vh;
  double c1 = cf->one_link, c3 = cf->three_staple, c5 = cf->five_staple, c7 = cf->seven_staple, cL = cf->lepage;
  c1 -= 6 * cL;
  bool have5 = c5 != 0 || c7 != 0 || cL != 0;
  bool have3 = c3 != 0 || have5;
  double2 *stp = dalloc<double2>(F), *tmp = dalloc<double2>(F);
  for (int dir = 0; dir < 4; dir++) {
    k_scale_field<<<grid_for(F, 256), 256, 0, ctx().s>>>(fl + dir * F, gf + dir * F, c1, F);
    QLAUNCH();
    if (!have3) continue;
    for (int nu = 0; nu < 4; nu++) {
      if (nu == dir) continue;
      staple(fl + dir * F, stp, gf + dir * F, gf + nu * F, dir, nu, c3);
      if (cL != 0) staple(fl + dir * F, nullptr, stp, gf + nu * F, dir, nu, cL);
      if (c5 != 0 || c7 != 0) {
        for (int rho = 0; rho < 4; rho++) {
          if (rho == dir || rho == nu) continue;
          staple(fl + dir * F, tmp, stp, gf + rho * F, dir, rho, c5);
          if (c7 != 0)
            for (int sig = 0; sig < 4; sig++)
              if (sig != dir && sig != nu && sig != rho) staple(fl + dir * F, nullptr, tmp, gf + sig * F, dir, sig, c7);
        }
      }
    }
  }
  if (ll) {
    for (int dir = 0; dir < 4; dir++) {
      k_naik<<<grid_for(2 * g.Vh, 128), 128, 0, ctx().s>>>(ll + dir * F, gfLong + dir * F, dir, cf->naik, g);
      QLAUNCH();
    }
  }
  dfree(stp); dfree(tmp);
  return (have3 || cf->naik != 0) ? 61632.0 * (double)g.V : 0.0;
}

// ---------------------------------------------------------------- U(3) projection
__device__ double2 det3(const M3 &u) {
  double2 m0 = csub<double>(cmul<double>(u.e[4], u.e[8]), cmul<double>(u.e[5], u.e[7]));
  double2 m1 = csub<double>(cmul<double>(u.e[3], u.e[8]), cmul<double>(u.e[5], u.e[6]));
  double2 m2 = csub<double>(cmul<double>(u.e[3], u.e[7]), cmul<double>(u.e[4], u.e[6]));
  double2 d = csub<double>(cmul<double>(u.e[0], m0), cmul<double>(u.e[1], m1));
  return cadd<double>(d, cmul<double>(u.e[2], m2));
}

struct ReunitOpt { int allow_svd, svd_only; double rel, abs; };

__device__ int u3_un_analytic(const M3 &V, M3 &W, const ReunitOpt o) {
  const double EPS = 1.0e-14, PI = 3.14159265358979323846;
  double det_check = 0;
  if (o.allow_svd) {
    double2 d = det3(V);
    det_check = d.x * d.x + d.y * d.y;
  }
  M3 Q = mul_an(V, V), Q2 = mul(Q, Q), Q3 = mul(Q2, Q);
  double c0 = Q.e[0].x + Q.e[4].x + Q.e[8].x;
  double c1 = (Q2.e[0].x + Q2.e[4].x + Q2.e[8].x) / 2;
  double c2 = (Q3.e[0].x + Q3.e[4].x + Q3.e[8].x) / 3;
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
  bool svd = false;
  if (o.allow_svd) {
    if (!o.svd_only) {
      if (det_check != 0 && fabs(det_check - g0 * g1 * g2) / fabs(det_check) > o.rel) svd = true;
      if (det_check < o.abs) svd = true;
    } else svd = true;
  }
  if (svd) {
    double w[3]; M3 Z, S2;
    herm_eig3(Q, w, Z);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        double2 s = make_double2(0, 0);
        for (int k = 0; k < 3; k++) {
          double f = w[k] > 0 ? 1.0 / sqrt(w[k]) : 0.0;
          double2 t = cmul<double>(Z.e[3 * i + k], make_double2(Z.e[3 * j + k].x, -Z.e[3 * j + k].y));
          s.x += f * t.x; s.y += f * t.y;
        }
        S2.e[3 * i + j] = s;
      }
    W = mul(V, S2);
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
  M3 S2;
  for (int e = 0; e < 9; e++) S2.e[e] = make_double2(f1 * Q.e[e].x + f2 * Q2.e[e].x, f1 * Q.e[e].y + f2 * Q2.e[e].y);
  S2.e[0].x += f0; S2.e[4].x += f0; S2.e[8].x += f0;
  W = mul(V, S2);
  return 0;
}

__global__ void k_u3reunit(double2 *W, const double2 *Vf, i64 Vh, ReunitOpt o, unsigned *nsvd) {
  i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;   // over [4][2][Vh]
  if (s >= 8 * Vh) return;
  i64 blk = s / Vh, i = s % Vh;
  const double2 *vb = Vf + blk * 9 * Vh + i;
  M3 V = ld3(vb, Vh), Wm;
  int k = u3_un_analytic(V, Wm, o);
  st3(W + blk * 9 * Vh + i, Vh, Wm);
  if (k) atomicAdd(nsvd, 1u);
}

// ---------------------------------------------------------------- link object
template <typename T, typename TS>
__global__ void k_load_fwd(c2<T> *lk, const c2<TS> *fat, const c2<TS> *lng, int nl, double sc, i64 Vh) {
  i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;   // over [2 p][4 mu][9 e][Vh]
  if (s >= 72 * Vh) return;
  i64 i = s % Vh, t = s / Vh;
  int e = (int)(t % 9), mu = (int)((t / 9) % 4), p = (int)(t / 36);
  i64 src = ((i64)mu * 18 + (i64)p * 9 + e) * Vh + i;
  int fs = nl == 16 ? 4 * mu : 2 * mu;
  c2<TS> v = fat[src];
  lk[(((i64)p * nl + fs) * 9 + e) * Vh + i] = mk<T>((T)(sc * v.x), (T)(sc * v.y));
  if (nl == 16) {
    c2<TS> w = lng[src];
    lk[(((i64)p * nl + fs + 1) * 9 + e) * Vh + i] = mk<T>((T)(sc * w.x), (T)(sc * w.y));
  }
}

template <typename T>
__global__ void k_extract_fwd(c2<T> *fat, c2<T> *lng, const c2<T> *lk, int nl, double sc, i64 Vh) {
  i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (s >= 72 * Vh) return;
  i64 i = s % Vh, t = s / Vh;
  int e = (int)(t % 9), mu = (int)((t / 9) % 4), p = (int)(t / 36);
  i64 dst = ((i64)mu * 18 + (i64)p * 9 + e) * Vh + i;
  int fs = nl == 16 ? 4 * mu : 2 * mu;
  c2<T> v = lk[(((i64)p * nl + fs) * 9 + e) * Vh + i];
  fat[dst] = mk<T>((T)(sc * v.x), (T)(sc * v.y));
  if (nl == 16 && lng) {
    c2<T> w = lk[(((i64)p * nl + fs + 1) * 9 + e) * Vh + i];
    lng[dst] = mk<T>((T)(sc * w.x), (T)(sc * w.y));
  }
}

// bck slot k at (p, x) = -fwd slot(k)(x - d mu)^+   (parity 1-p)
template <typename T>
__global__ void k_double_store(c2<T> *lk, int nl, Geom g) {
  i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;   // over [2][nl/2][Vh]
  const i64 Vh = g.Vh;
  const int nb = nl / 2;
  if (s >= 2 * nb * Vh) return;
  int i = (int)(s % Vh), t = (int)(s / Vh);
  int b = t % nb, p = t / nb;
  int k, kf, mu, d;
  if (nl == 16) { mu = b / 2; k = 4 * mu + 2 + (b & 1); kf = k - 2; d = (b & 1) ? 3 : 1; }
  else { mu = b; k = 2 * mu + 1; kf = k - 1; d = 1; }
  int x[4];
  site_coords(g, i, p, x);
  int j = nbr_index(g, x, mu, -d);
  const c2<T> *F = lk + (((i64)(1 - p) * nl + kf) * 9) * Vh + j;
  c2<T> *B = lk + (((i64)p * nl + k) * 9) * Vh + i;
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      c2<T> v = F[(3 * c + a) * Vh];
      B[(3 * a + c) * Vh] = mk<T>(-v.x, v.y);
    }
}

// rephase_L (asqtad_dslash_p.c:1385-1446): boundary phase on the last slice
// (fat) or last three slices (long), staggered sign from r0-shifted coords
template <typename T>
__global__ void k_rephase_L(c2<T> *lk, int nl, Geom g, int dir, int bc_dir, double phr, double phi, int bits,
                            int4 r0) {
  i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;   // over [2][2 kinds][Vh]
  const i64 Vh = g.Vh;
  if (s >= 4 * Vh) return;
  int i = (int)(s % Vh), t = (int)(s / Vh);
  int kind = t & 1, p = t >> 1;
  if (kind == 1 && nl != 16) return;
  int x[4];
  site_coords(g, i, p, x);
  for (int j = 0; j < 4; j++) x[j] += g.O[j];   // global coordinates
  const int r0a[4] = {r0.x, r0.y, r0.z, r0.w};
  double fr = 1, fi = 0;
  if (bc_dir >= 0) {
    int n = g.GL[bc_dir];
    int rshift = (x[bc_dir] + n - r0a[bc_dir]) % n;
    bool hit = kind == 0 ? (rshift == n - 1) : (rshift >= n - 3);
    if (hit) { fr = phr; fi = phi; }
  }
  if (bits) {
    int sgn = 0;
    for (int j = 0; j < 4; j++) {
      int n = g.GL[j];
      sgn += ((bits >> j) & 1) * ((x[j] + n - r0a[j]) % n);
    }
    if (sgn & 1) { fr = -fr; fi = -fi; }
  }
  if (fr == 1 && fi == 0) return;
  int k = nl == 16 ? 4 * dir + kind : 2 * dir;
  c2<T> *B = lk + (((i64)p * nl + k) * 9) * Vh + i;
  for (int e = 0; e < 9; e++) {
    c2<T> v = B[e * Vh];
    B[e * Vh] = mk<T>((T)(fr * v.x - fi * v.y), (T)(fr * v.y + fi * v.x));
  }
}

template <typename T>
FlaT<T> *fla_alloc(int nlinks) {
  const Geom &g = ctx().g;
  FlaT<T> *f = new FlaT<T>();
  f->nlinks = nlinks;
  f->d = dalloc<c2<T>>(2LL * nlinks * 9 * g.Vh);
  handle_register(f);
  return f;
}

template <typename T>
void double_store(FlaT<T> *f) {
  const Geom &g = ctx().g;
  i64 n = 2LL * (f->nlinks / 2) * g.Vh;
  k_double_store<T><<<grid_for(n, 256), 256, 0, ctx().s>>>(f->d, f->nlinks, g);
  QLAUNCH();
}

template <typename T>
void fla_load_fwd(FlaT<T> *f, const c2<T> *fat, const c2<T> *lng, double scale) {
  const Geom &g = ctx().g;
  k_load_fwd<T, T><<<grid_for(72 * g.Vh, 256), 256, 0, ctx().s>>>(f->d, fat, lng, f->nlinks, scale, g.Vh);
  QLAUNCH();
  double_store(f);
}

template <typename T>
void fla_extract_fwd(FlaT<T> *f, c2<T> *fat, c2<T> *lng, double scale) {
  const Geom &g = ctx().g;
  k_extract_fwd<T><<<grid_for(72 * g.Vh, 256), 256, 0, ctx().s>>>(fat, lng, f->d, f->nlinks, scale, g.Vh);
  QLAUNCH();
}

template <typename T>
void fla_rephase(FlaT<T> *f, const int *r0, const QOP_Complex *bc, const int *sign) {
  const Geom &g = ctx().g;
  int4 r = make_int4(r0 ? r0[0] : 0, r0 ? r0[1] : 0, r0 ? r0[2] : 0, r0 ? r0[3] : 0);
  for (int i = 0; i < 4; i++) {
    int bc_dir = -1;
    double pr = 1, pi = 0;
    if (bc && (bc[i].re != 1. || bc[i].im != 0.)) { bc_dir = i; pr = bc[i].re; pi = bc[i].im; }
    int bits = sign ? sign[i] : 0;
    if (!sign && bc_dir < 0) continue;
    k_rephase_L<T><<<grid_for(4 * g.Vh, 256), 256, 0, ctx().s>>>(f->d, f->nlinks, g, i, bc_dir, pr, pi, bits, r);
    QLAUNCH();
  }
  double_store(f);
}

template <typename T>
void fla_destroy(FlaT<T> *f) {
  if (!f) return;
  sloppy_invalidate((void *)f);
  if (f->eigcg && f->eigcg_free) f->eigcg_free(f->eigcg);
  dfree(f->d);
  handle_forget(f);
  delete f;
}

template <typename TD, typename TS>
__global__ void k_conv_links(c2<TD> *d, const c2<TS> *s, double sc, i64 n) {
  i64 k = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (k >= n) return;
  c2<TS> v = s[k];
  d[k] = mk<TD>((TD)(sc * v.x), (TD)(sc * v.y));
}

// QOP_FD_asqtad_create_L_from_L / create_L_from_r_times_L
// (asqtad_dslash_p.c:700-910): negation, conjugation and transposition are
// exact, so scaling or rounding every slot equals re-double-storing
template <typename TD, typename TS>
FlaT<TD> *fla_convert(FlaT<TS> *src) {
  const Geom &g = ctx().g;
  FlaT<TD> *f = fla_alloc<TD>(src->nlinks);
  i64 n = 2LL * src->nlinks * 9 * g.Vh;
  k_conv_links<TD, TS><<<grid_for(n, 256), 256, 0, ctx().s>>>(f->d, src->d, 1.0, n);
  QLAUNCH();
  return f;
}

template <typename T>
FlaT<T> *fla_scaled_copy(FlaT<T> *src, double s) {
  const Geom &g = ctx().g;
  FlaT<T> *f = fla_alloc<T>(src->nlinks);
  i64 n = 2LL * src->nlinks * 9 * g.Vh;
  k_conv_links<T, T><<<grid_for(n, 256), 256, 0, ctx().s>>>(f->d, src->d, s, n);
  QLAUNCH();
  return f;
}

template <typename T>
__global__ void k_add_links(c2<T> *d, const c2<T> *s, i64 n) {
  i64 k = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (k >= n) return;
  c2<T> a = d[k], b = s[k];
  d[k] = mk<T>(a.x + b.x, a.y + b.y);
}

// QOP_asqtad_L_peq_L (asqtad_dslash_p.c:912-925): fat += fat, long += long
template <typename T>
void fla_peq(FlaT<T> *f, FlaT<T> *h) {
  const Geom &g = ctx().g;
  if (f->nlinks == h->nlinks) {
    i64 n = 2LL * f->nlinks * 9 * g.Vh;
    k_add_links<T><<<grid_for(n, 256), 256, 0, ctx().s>>>(f->d, h->d, n);
    QLAUNCH();
    return;
  }
  // one of them has no Naik links: add the fat parts slot by slot
  for (int p = 0; p < 2; p++)
    for (int mu = 0; mu < 4; mu++) {
      int kf = f->nlinks == 16 ? 4 * mu : 2 * mu, kh = h->nlinks == 16 ? 4 * mu : 2 * mu;
      i64 n = 9 * g.Vh;
      k_add_links<T><<<grid_for(n, 256), 256, 0, ctx().s>>>(f->d + ((i64)p * f->nlinks + kf) * 9 * g.Vh,
                                                           h->d + ((i64)p * h->nlinks + kh) * 9 * g.Vh, n);
      QLAUNCH();
    }
  double_store(f);
}

// asqtad links from one or two FP64 gauge fields ([4][2][9][Vh])
template <typename T>
static FlaT<T> *fla_from_fields(const double2 *fat, const double2 *lng) {
  const Geom &g = ctx().g;
  FlaT<T> *f = fla_alloc<T>(lng ? 16 : 8);
  k_load_fwd<T, double><<<grid_for(72 * g.Vh, 256), 256, 0, ctx().s>>>(f->d, fat, lng, f->nlinks, 0.5, g.Vh);
  QLAUNCH();
  double_store(f);
  return f;
}

template <typename T>
double2 *gauge_fp64(GaugeT<T> *G, bool &owned) {
  const Geom &g = ctx().g;
  if (std::is_same<T, double>::value) { owned = false; return (double2 *)G->d; }
  owned = true;
  i64 n = 72 * g.Vh;
  double2 *d = dalloc<double2>(n);
  convert<double, T>(d, G->d, Range{0, n});
  return d;
}
template double2 *gauge_fp64<float>(GaugeT<float> *, bool &);
template double2 *gauge_fp64<double>(GaugeT<double> *, bool &);

template <typename T>
FlaT<T> *fla_from_G(QOP_info_t *info, const QOP_asqtad_coeffs_t *coef, GaugeT<T> *gfat, GaugeT<T> *glong) {
  dd_refuse("asqtad_create_L_from_G");   // staples reach across the block faces
  const Geom &g = ctx().g;
  double t0 = wtime();
  bool o1, o2 = false;
  double2 *gf = gauge_fp64(gfat, o1);
  double2 *gl = (glong && glong != gfat) ? gauge_fp64(glong, o2) : gf;
  const i64 F4 = 72 * g.Vh;
  double2 *fl = dalloc<double2>(F4), *ll = coef->naik != 0 ? dalloc<double2>(F4) : nullptr;
  double flop = make_imp_links(coef, gf, gl, fl, ll);
  FlaT<T> *f = fla_from_fields<T>(fl, ll);
  dfree(fl); if (ll) dfree(ll);
  if (o1) dfree(gf);
  if (o2) dfree(gl);
  sync();
  if (info) { info->final_sec = wtime() - t0; info->final_flop = flop; info->status = QOP_SUCCESS; }
  return f;
}

// hisq_links_p.c:62-256 with the reference's coefficient mapping
template <typename T>
HisqT<T> *hisq_from_G(QOP_info_t *info, const QOP_hisq_coeffs_t *c, GaugeT<T> *gauge) {
  dd_refuse("hisq_create_L_from_G");
  const Geom &g = ctx().g;
  const Options &o = ctx().opt;
  double t0 = wtime(), flop = 0;
  if (c->ugroup == QOP_UNITARIZE_SU3) fail(QOP_FAIL, "hisq_create_L_from_G: SU(3) projection is not supported");
  if (c->n_naiks < 1 || c->n_naiks > QOP_MAX_NAIK) fail(QOP_FAIL, "hisq_create_L_from_G: bad n_naiks %d", c->n_naiks);
  QOP_asqtad_coeffs_t a1{}, a2{}, a3{};
  a1.one_link = c->fat7_one_link; a1.three_staple = c->fat7_three_staple;
  a1.five_staple = c->fat7_five_staple; a1.seven_staple = c->fat7_seven_staple;
  a1.lepage = o.use_fat7_lepage ? c->fat7_lepage : 0.0; a1.naik = 0;
  a2.one_link = c->asqtad_one_link; a2.three_staple = c->asqtad_three_staple;
  a2.five_staple = c->asqtad_five_staple; a2.seven_staple = c->asqtad_seven_staple;
  a2.lepage = c->asqtad_lepage; a2.naik = c->asqtad_naik;
  a3.one_link = c->difference_one_link; a3.naik = c->difference_naik;
  HisqT<T> *h = new HisqT<T>();
  handle_register(h);
  h->n_naiks = c->n_naiks;
  bool own;
  double2 *U = gauge_fp64(gauge, own);
  const i64 F4 = 72 * g.Vh;
  double2 *Vl = dalloc<double2>(F4), *Wl = dalloc<double2>(F4);
  // fat7 stage (the reference's x1/2 on load and x2 afterwards cancel)
  flop += make_imp_links(&a1, U, U, Vl, nullptr);
  flop += 198.0 * g.V;
  // U(3) projection
  unsigned *d_nsvd = dalloc<unsigned>(1);
  dzero(d_nsvd, sizeof(unsigned));
  ReunitOpt ro{o.reunit_allow_svd, o.reunit_svd_only, o.reunit_svd_rel_error, o.reunit_svd_abs_error};
  k_u3reunit<<<grid_for(8 * g.Vh, 128), 128, 0, ctx().s>>>(Wl, Vl, g.Vh, ro, d_nsvd);
  QLAUNCH();
  unsigned nsvd = 0;
  QCHECK(cudaMemcpyAsync(&nsvd, d_nsvd, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx().s));
  sync();
  dfree(d_nsvd);
  flop += 795.0 * 4 * g.V;
  // asqtad stage on the projected links
  auto stage = [&](const QOP_asqtad_coeffs_t *cf) {
    double2 *fl = dalloc<double2>(F4), *ll = cf->naik != 0 ? dalloc<double2>(F4) : nullptr;
    flop += make_imp_links(cf, Wl, Wl, fl, ll);
    FlaT<T> *f = fla_from_fields<T>(fl, ll);
    dfree(fl); if (ll) dfree(ll);
    return f;
  };
  if (c->n_naiks > 1) {
    FlaT<T> *d = stage(&a3);
    if (o.want_deps) h->fn_deps = fla_scaled_copy<T>(d, 1.0);
    for (int k = 1; k < c->n_naiks; k++) h->fn[k] = fla_scaled_copy<T>(d, c->eps_naik[k]);
    fla_destroy(d);
    h->fn[0] = stage(&a2);
    for (int k = 1; k < c->n_naiks; k++) fla_peq<T>(h->fn[k], h->fn[0]);
  } else {
    h->fn[0] = stage(&a2);
    if (o.want_deps) h->fn_deps = stage(&a3);
  }
  if (o.want_aux) {
    h->U = gauge_new<T>(); h->V = gauge_new<T>(); h->W = gauge_new<T>();
    convert<T, double>(h->U->d, U, Range{0, F4});
    convert<T, double>(h->V->d, Vl, Range{0, F4});
    convert<T, double>(h->W->d, Wl, Range{0, F4});
  }
  dfree(Vl); dfree(Wl);
  if (own) dfree(U);
  sync();
  if (info) {
    info->final_sec = wtime() - t0;
    info->final_flop = flop;
    info->status = QOP_SUCCESS;
    info->count1 += (int)nsvd;
  }
  return h;
}

template <typename T>
void hisq_destroy(HisqT<T> *h) {
  if (!h) return;
  for (int k = 0; k < h->n_naiks; k++) fla_destroy(h->fn[k]);
  fla_destroy(h->fn_deps);
  gauge_destroy(h->U); gauge_destroy(h->V); gauge_destroy(h->W);
  handle_forget(h);
  delete h;
}

#define INST(T)                                                                                     \
  template FlaT<T> *fla_alloc<T>(int);                                                              \
  template void double_store<T>(FlaT<T> *);                                                         \
  template void fla_load_fwd<T>(FlaT<T> *, const c2<T> *, const c2<T> *, double);                  \
  template void fla_extract_fwd<T>(FlaT<T> *, c2<T> *, c2<T> *, double);                            \
  template void fla_rephase<T>(FlaT<T> *, const int *, const QOP_Complex *, const int *);           \
  template void fla_destroy<T>(FlaT<T> *);                                                          \
  template FlaT<T> *fla_scaled_copy<T>(FlaT<T> *, double);                                          \
  template void fla_peq<T>(FlaT<T> *, FlaT<T> *);                                                   \
  template FlaT<T> *fla_from_G<T>(QOP_info_t *, const QOP_asqtad_coeffs_t *, GaugeT<T> *, GaugeT<T> *); \
  template HisqT<T> *hisq_from_G<T>(QOP_info_t *, const QOP_hisq_coeffs_t *, GaugeT<T> *);          \
  template void hisq_destroy<T>(HisqT<T> *);
INST(float)
INST(double)
template FlaT<float> *fla_convert<float, double>(FlaT<double> *);
template FlaT<double> *fla_convert<double, float>(FlaT<float> *);

}  // namespace qopb
