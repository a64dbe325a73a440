// force.cu -- asqtad fermion force on the device.
// Reference: lib/asqtad_force_p.c:16-64 (QOP_asqtad_force / _multi),
// lib/asqtad_force_fnmat_p.c:4-43 (outer products of the sources, scale -1),
// :491-513 (sign flip on odd sites), :516-546 (force += -2 antiherm(U deriv^+)).
//
// deriv_mu is the derivative of
//   E(U) = Re sum_{x,mu} tr[ midF_mu(x)^+ fat_mu(x) + midN_mu(x)^+ long_mu(x) ]
// with (fat, long) = make_imp_links(U), in the convention
// dE = Re sum tr[deriv^+ dU].  It is formed by reverse-mode differentiation
// of the staple sums of make_imp_links (links.cu): for every staple
// application out += c staple(in; mu, nu) the adjoint kernels add the
// contributions to the adjoint of `in` and of U_nu, in the reverse order of
// the forward sums (7-staples, 5-staples, Lepage, 3-staples, one-link), and
// the Naik products add theirs.  Every adjoint kernel is written in gather
// form (each thread owns one output site and reads its neighbours), so no
// atomics are needed and results are deterministic.  Everything runs in
// FP64; the result is rounded once into the force handle's precision.
#include "fields.cuh"
#include "mat3.cuh"
#include <vector>

namespace qopb {
namespace {

__device__ __forceinline__ void site_of(const Geom &g, i64 s, int &p, int &i, int x[4]) {
  p = (int)(s / g.Vh);
  i = (int)(s % g.Vh);
  site_coords(g, i, p, x);
}
__device__ __forceinline__ void nbr_pi(const Geom &g, const int x[4], int mu, int d, int &p, int &i) {
  int y[4];
  shifted(g, x, mu, d, y);
  par_idx(g, y, p, i);
}
__device__ __forceinline__ M3 ldf(const double2 *f, const Geom &g, int p, int i) { return ld3(fptr(f, g, p, i), g.Vh); }
__device__ __forceinline__ void accf(double2 *f, const Geom &g, int p, int i, const M3 &m, double c) {
  double2 *b = f + (i64)p * 9 * g.Vh + i;
#pragma unroll
  for (int e = 0; e < 9; e++) {
    double2 v = b[e * g.Vh];
    b[e * g.Vh] = make_double2(v.x + c * m.e[e].x, v.y + c * m.e[e].y);
  }
}

// out = staple(in; mu, nu) = U_nu(x) in(x+nu) U_nu(x+mu)^+ + U_nu(y)^+ in(y) U_nu(y+mu), y = x-nu
__global__ void k_fstaple(double2 *out, const double2 *in, const double2 *Unu, int mu, int nu, Geom g) {
  const i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (s >= 2 * g.Vh) return;
  int p, i, x[4], pn, in_, pm, im, py, iy, pym, iym, yy[4];
  site_of(g, s, p, i, x);
  nbr_pi(g, x, nu, 1, pn, in_);
  nbr_pi(g, x, mu, 1, pm, im);
  shifted(g, x, nu, -1, yy);
  par_idx(g, yy, py, iy);
  nbr_pi(g, yy, mu, 1, pym, iym);
  M3 up = mul(ldf(Unu, g, p, i), mul_na(ldf(in, g, pn, in_), ldf(Unu, g, pm, im)));
  M3 lo = mul(mul_an(ldf(Unu, g, py, iy), ldf(in, g, py, iy)), ldf(Unu, g, pym, iym));
#pragma unroll
  for (int e = 0; e < 9; e++) up.e[e] = make_double2(up.e[e].x + lo.e[e].x, up.e[e].y + lo.e[e].y);
  st3(out + (i64)p * 9 * g.Vh + i, g.Vh, up);
}

// adjoint of `in` for out += c staple(in; mu, nu):
// Gin(z) += c [U_nu(z-nu)^+ G(z-nu) U_nu(z-nu+mu) + U_nu(z) G(z+nu) U_nu(z+mu)^+]
__global__ void k_adj_in(double2 *Gin, const double2 *G, const double2 *Unu, int mu, int nu, double c, Geom g) {
  const i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (s >= 2 * g.Vh) return;
  int p, i, z[4], a, ai, b, bi, pn, in_, pm, im, y[4];
  site_of(g, s, p, i, z);
  shifted(g, z, nu, -1, y);
  par_idx(g, y, a, ai);                 // z - nu
  nbr_pi(g, y, mu, 1, b, bi);           // z - nu + mu
  nbr_pi(g, z, nu, 1, pn, in_);         // z + nu
  nbr_pi(g, z, mu, 1, pm, im);          // z + mu
  M3 r = mul(mul_an(ldf(Unu, g, a, ai), ldf(G, g, a, ai)), ldf(Unu, g, b, bi));
  accf(Gin, g, p, i, r, c);
  r = mul_na(mul(ldf(Unu, g, p, i), ldf(G, g, pn, in_)), ldf(Unu, g, pm, im));
  accf(Gin, g, p, i, r, c);
}

// adjoint of U_nu for out += c staple(in; mu, nu):
// GU(z) += c [G(z) U(z+mu) in(z+nu)^+ + G(z-mu)^+ U(z-mu) in(z-mu+nu)
//             + in(z-mu)^+ U(z-mu) G(z-mu+nu) + in(z) U(z+mu) G(z+nu)^+],  U = U_nu
__global__ void k_adj_link(double2 *GU, const double2 *G, const double2 *in, const double2 *Unu, int mu, int nu,
                           double c, Geom g) {
  const i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (s >= 2 * g.Vh) return;
  int p, i, z[4], pm, im, pn, in_, qm, iqm, qmn, iqmn, y[4];
  site_of(g, s, p, i, z);
  nbr_pi(g, z, mu, 1, pm, im);          // z + mu
  nbr_pi(g, z, nu, 1, pn, in_);         // z + nu
  shifted(g, z, mu, -1, y);
  par_idx(g, y, qm, iqm);               // z - mu
  nbr_pi(g, y, nu, 1, qmn, iqmn);       // z - mu + nu
  const M3 Upm = ldf(Unu, g, pm, im), Uqm = ldf(Unu, g, qm, iqm);
  M3 r = mul_na(mul(ldf(G, g, p, i), Upm), ldf(in, g, pn, in_));
  accf(GU, g, p, i, r, c);
  r = mul(mul_an(ldf(G, g, qm, iqm), Uqm), ldf(in, g, qmn, iqmn));
  accf(GU, g, p, i, r, c);
  r = mul(mul_an(ldf(in, g, qm, iqm), Uqm), ldf(G, g, qmn, iqmn));
  accf(GU, g, p, i, r, c);
  r = mul_na(mul(ldf(in, g, p, i), Upm), ldf(G, g, pn, in_));
  accf(GU, g, p, i, r, c);
}

// adjoint of long(x) = c U(x) U(x+mu) U(x+2mu):
// D(z) += c [N(z) (U(z+mu) U(z+2mu))^+ + U(z-mu)^+ N(z-mu) U(z+mu)^+ + (U(z-2mu) U(z-mu))^+ N(z-2mu)]
__global__ void k_adj_naik(double2 *D, const double2 *N, const double2 *U, int mu, double c, Geom g) {
  const i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (s >= 2 * g.Vh) return;
  int p, i, z[4], p1, i1, p2, i2, m1, j1, m2, j2;
  site_of(g, s, p, i, z);
  nbr_pi(g, z, mu, 1, p1, i1);
  nbr_pi(g, z, mu, 2, p2, i2);
  nbr_pi(g, z, mu, -1, m1, j1);
  nbr_pi(g, z, mu, -2, m2, j2);
  const M3 Up1 = ldf(U, g, p1, i1), Um1 = ldf(U, g, m1, j1);
  M3 r = mul_na(ldf(N, g, p, i), mul(Up1, ldf(U, g, p2, i2)));
  accf(D, g, p, i, r, c);
  r = mul_na(mul_an(Um1, ldf(N, g, m1, j1)), Up1);
  accf(D, g, p, i, r, c);
  r = mul_an(mul(ldf(U, g, m2, j2), Um1), ldf(N, g, m2, j2));
  accf(D, g, p, i, r, c);
}

// The reference's derivative field carries, with a Lepage term, one more
// term of the form U_mu H, H Hermitian (lib/asqtad_force_fnmat_p.c:316-340):
//   D_mu(x) -= cL [F_mu(x) U_mu(x) - U_mu(x) F_mu(x+mu)],
//   F_mu = sum_{nu != mu} H_nu,  H_nu = A_nu + A_nu^+,
//   A_nu(x) = M_nu(x) U_nu(x)^+ - M_nu(x-nu)^+ U_nu(x-nu).
// The force projection TA(U D^+) removes it; the filtered U(3) adjoint of
// the HISQ force, which receives this field at the W level, does not.
// k_lep_h: H = H_nu for one nu
__global__ void k_lep_h(double2 *H, const double2 *M, const double2 *Unu, int nu, Geom g) {
  const i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (s >= 2 * g.Vh) return;
  int p, i, z[4], pm, im;
  site_of(g, s, p, i, z);
  nbr_pi(g, z, nu, -1, pm, im);
  const M3 a = mul_na(ldf(M, g, p, i), ldf(Unu, g, p, i));
  const M3 b = mul_an(ldf(M, g, pm, im), ldf(Unu, g, pm, im));
  M3 h;
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double2 x = a.e[3 * r + c], y = b.e[3 * r + c], xt = a.e[3 * c + r], yt = b.e[3 * c + r];
      h.e[3 * r + c] = make_double2(x.x - y.x + xt.x - yt.x, x.y - y.y - xt.y + yt.y);
    }
  st3(H + (i64)p * 9 * g.Vh + i, g.Vh, h);
}

// k_lep_fix: D_mu -= cL [F U_mu - U_mu F(x+mu)] with F the sum of the three
// H_nu (nu != mu) given in h0..h2
__global__ void k_lep_fix(double2 *D, const double2 *Umu, const double2 *h0, const double2 *h1, const double2 *h2,
                          int mu, double cL, Geom g) {
  const i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (s >= 2 * g.Vh) return;
  int p, i, z[4], pp, ip;
  site_of(g, s, p, i, z);
  nbr_pi(g, z, mu, 1, pp, ip);
  M3 f0 = ldf(h0, g, p, i), f1 = ldf(h0, g, pp, ip);
  const M3 a0 = ldf(h1, g, p, i), a1 = ldf(h1, g, pp, ip), b0 = ldf(h2, g, p, i), b1 = ldf(h2, g, pp, ip);
#pragma unroll
  for (int e = 0; e < 9; e++) {
    f0.e[e] = make_double2(f0.e[e].x + a0.e[e].x + b0.e[e].x, f0.e[e].y + a0.e[e].y + b0.e[e].y);
    f1.e[e] = make_double2(f1.e[e].x + a1.e[e].x + b1.e[e].x, f1.e[e].y + a1.e[e].y + b1.e[e].y);
  }
  const M3 U = ldf(Umu, g, p, i);
  M3 r = mul(f0, U);
  const M3 t = mul(U, f1);
#pragma unroll
  for (int e = 0; e < 9; e++) r.e[e] = make_double2(r.e[e].x - t.e[e].x, r.e[e].y - t.e[e].y);
  accf(D, g, p, i, r, -cL);
}

__global__ void k_field_axpby(double2 *d, double a, const double2 *s, double b, i64 n) {   // d = a d + b s
  const i64 k = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double2 x = d[k], y = s[k];
  d[k] = make_double2(a * x.x + b * y.x, a * x.y + b * y.y);
}

// midF_mu(x) = sgn(x) sum_i eps_i x_i(x) x_i(x+mu)^+ (midN: x+3mu) with
// sgn = even_sign on even and -even_sign on odd sites (asqtad: -1, HISQ: +1);
// vectors are [parity][colour][site]
template <typename T>
__global__ void k_force_mid(double2 *midF, double2 *midN, const c2<T> *const *xs, const double *eps, int nsrc,
                            double even_sign, Geom g) {
  const i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (s >= 2 * g.Vh) return;
  int p, i, x[4];
  site_of(g, s, p, i, x);
  const double sgn = p ? -even_sign : even_sign;
  const i64 Vh = g.Vh;
  for (int mu = 0; mu < 4; mu++) {
    for (int k = 0; k < 2; k++) {
      double2 *out = k == 0 ? midF : midN;
      if (!out) continue;
      int q, j;
      nbr_pi(g, x, mu, k == 0 ? 1 : 3, q, j);
      M3 m;
#pragma unroll
      for (int e = 0; e < 9; e++) m.e[e] = make_double2(0, 0);
      for (int n = 0; n < nsrc; n++) {
        const c2<T> *v = xs[n];
        const double w = sgn * eps[n];
        double2 a[3], b[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const c2<T> va = v[((i64)p * 3 + c) * Vh + i], vb = v[((i64)q * 3 + c) * Vh + j];
          a[c] = make_double2((double)va.x, (double)va.y);
          b[c] = make_double2((double)vb.x, (double)vb.y);
        }
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
          for (int c = 0; c < 3; c++) {   // a_r conj(b_c)
            m.e[3 * r + c].x += w * (a[r].x * b[c].x + a[r].y * b[c].y);
            m.e[3 * r + c].y += w * (a[r].y * b[c].x - a[r].x * b[c].y);
          }
      }
      st3(out + (i64)mu * 18 * Vh + (i64)p * 9 * Vh + i, Vh, m);
    }
  }
}

// F_mu(x) = TA(F_mu(x)): the projection the reference's ASVEC algorithm
// applies to the whole accumulated force (lib/asqtad_force_asvec_p.c:403-408)
template <typename T>
__global__ void k_force_ta_self(c2<T> *F, Geom g) {
  const i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (s >= 8 * g.Vh) return;           // [4 mu][2 parities][Vh]
  const i64 Vh = g.Vh;
  const i64 off = (s / Vh) * 9 * Vh + s % Vh;
  double2 a[9];
#pragma unroll
  for (int e = 0; e < 9; e++) {
    const c2<T> v = F[off + (i64)e * Vh];
    a[e] = make_double2((double)v.x, (double)v.y);
  }
  double tri = 0;
#pragma unroll
  for (int k = 0; k < 3; k++) tri += a[4 * k].y;
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double2 x = a[3 * r + c], y = a[3 * c + r];
      double re = 0.5 * (x.x - y.x), im = 0.5 * (x.y + y.y);
      if (r == c) im -= tri / 3.0;
      c2<T> &f = F[off + (i64)(3 * r + c) * Vh];
      f.x = (T)re;
      f.y = (T)im;
    }
}

// F_mu(x) += fac TA(U_mu(x) D_mu(x)^+), TA = traceless anti-Hermitian part
template <typename T>
__global__ void k_force_ta(c2<T> *F, const double2 *U, const double2 *D, double fac, Geom g) {
  const i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (s >= 8 * g.Vh) return;           // [4 mu][2 parities][Vh]
  const i64 Vh = g.Vh;
  const i64 pm = s / Vh, i = s % Vh;   // pm = mu * 2 + parity
  const i64 off = pm * 9 * Vh + i;
  const M3 a = mul_na(ld3(U + off, Vh), ld3(D + off, Vh));
  double tri = 0;   // Im tr(a - a^+) / 2 = Im tr a
#pragma unroll
  for (int k = 0; k < 3; k++) tri += a.e[4 * k].y;
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double2 x = a.e[3 * r + c], y = a.e[3 * c + r];
      double re = 0.5 * (x.x - y.x), im = 0.5 * (x.y + y.y);
      if (r == c) im -= tri / 3.0;
      c2<T> &f = F[off + (i64)(3 * r + c) * Vh];
      f.x = (T)((double)f.x + fac * re);
      f.y = (T)((double)f.y + fac * im);
    }
}

// adjoint of the U(3) projection W = V f(Q), Q = V^+V, f(q) = q^-1/2:
// GV = GW f + V (B + B^+),  B = Z [(Z^+ V^+ GW Z) o Gamma] Z^+,
// Gamma_ij = (f(w_i) - f(w_j)) / (w_i - w_j) = -1 / (s_i s_j (s_i + s_j)), s = sqrt(w).
// Force filter (lib/hisq_reunit_utilities_p.c:463-481): where the smallest
// eigenvalue of Q is below ff, the derivative is the one of V (Q + ff)^-1/2.
__global__ void k_reunit_adj(double2 *GV, const double2 *V, const double2 *GW, i64 n4, double ff) {
  const i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;   // over [4 mu][2 parities][Vh]
  if (s >= n4) return;
  const i64 Vh = n4 / 8, blk = s / Vh, i = s % Vh, off = blk * 9 * Vh + i;
  const M3 v = ld3(V + off, Vh), gw = ld3(GW + off, Vh);
  M3 Z;
  double w[3], sq[3];
  herm_eig3(mul_an(v, v), w, Z);
  if (ff > 0 && fmin(w[0], fmin(w[1], w[2])) < ff) {
#pragma unroll
    for (int k = 0; k < 3; k++) w[k] += ff;
  }
#pragma unroll
  for (int k = 0; k < 3; k++) sq[k] = sqrt(w[k]);
  M3 f;
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      double2 acc = make_double2(0, 0);
#pragma unroll
      for (int k = 0; k < 3; k++) {   // Z_ak conj(Z_bk) / s_k
        const double2 za = Z.e[3 * a + k], zb = Z.e[3 * b + k];
        acc.x += (za.x * zb.x + za.y * zb.y) / sq[k];
        acc.y += (za.y * zb.x - za.x * zb.y) / sq[k];
      }
      f.e[3 * a + b] = acc;
    }
  M3 At = mul(mul_an(Z, mul_an(v, gw)), Z);
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      const double gm = -1.0 / (sq[a] * sq[b] * (sq[a] + sq[b]));
      At.e[3 * a + b] = make_double2(gm * At.e[3 * a + b].x, gm * At.e[3 * a + b].y);
    }
  const M3 B = mul_na(mul(Z, At), Z);
  M3 t;
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++)
      t.e[3 * a + b] = make_double2(B.e[3 * a + b].x + B.e[3 * b + a].x, B.e[3 * a + b].y - B.e[3 * b + a].y);
  M3 r = mul(gw, f);
  const M3 u = mul(v, t);
#pragma unroll
  for (int e = 0; e < 9; e++) r.e[e] = make_double2(r.e[e].x + u.e[e].x, r.e[e].y + u.e[e].y);
  st3(GV + off, Vh, r);
}

// Work fields of the reverse sweep ([2][9][Vh] each)
struct SweepWork {
  double2 *S3, *S5, *G3, *G5;
};

// D += derivative of Re sum tr[midF^+ fat + midN^+ long] with (fat, long) =
// make_imp_links(c, U): the reverse sweep over its staple sums and the Naik
// products; midN may be null.  lepage_rep adds the reference's Lepage term
// of the form U H (k_lep_h), for a derivative that feeds something other
// than the force projection.  Returns the number of kernels launched.
int smear_adjoint(const double2 *U, const double c[6], const double2 *mid, const double2 *midN, double2 *D,
                  const SweepWork &w, bool lepage_rep = false) {
  Context &cx = ctx();
  const Geom &g = cx.g;
  const i64 F1 = 18 * g.Vh;
  const int grid2 = grid_for(2 * g.Vh, 128), gridF = grid_for(F1, 256);
  const double c1 = c[0] - 6 * c[4], c3 = c[1], c5 = c[2], c7 = c[3], cL = c[4];
  const bool have5 = c5 != 0 || c7 != 0 || cL != 0, have3 = c3 != 0 || have5;
  auto Uf = [&](int d) { return U + d * F1; };
  auto Df = [&](int d) { return D + d * F1; };
  int nk = 0;
  for (int mu = 0; mu < 4; mu++) {
    const double2 *M = mid + mu * F1;
    k_field_axpby<<<gridF, 256, 0, cx.s>>>(Df(mu), 1.0, M, c1, F1);
    nk++;
    if (!have3) continue;
    for (int nu = 0; nu < 4; nu++) {
      if (nu == mu) continue;
      k_fstaple<<<grid2, 128, 0, cx.s>>>(w.S3, Uf(mu), Uf(nu), mu, nu, g);
      k_field_axpby<<<gridF, 256, 0, cx.s>>>(w.G3, 0.0, M, c3, F1);
      nk += 2;
      if (cL != 0) {
        k_adj_in<<<grid2, 128, 0, cx.s>>>(w.G3, M, Uf(nu), mu, nu, cL, g);
        k_adj_link<<<grid2, 128, 0, cx.s>>>(Df(nu), M, w.S3, Uf(nu), mu, nu, cL, g);
        nk += 2;
      }
      if (c5 != 0 || c7 != 0) {
        for (int rho = 0; rho < 4; rho++) {
          if (rho == mu || rho == nu) continue;
          k_fstaple<<<grid2, 128, 0, cx.s>>>(w.S5, w.S3, Uf(rho), mu, rho, g);
          k_field_axpby<<<gridF, 256, 0, cx.s>>>(w.G5, 0.0, M, c5, F1);
          nk += 2;
          if (c7 != 0)
            for (int sig = 0; sig < 4; sig++) {
              if (sig == mu || sig == nu || sig == rho) continue;
              k_adj_in<<<grid2, 128, 0, cx.s>>>(w.G5, M, Uf(sig), mu, sig, c7, g);
              k_adj_link<<<grid2, 128, 0, cx.s>>>(Df(sig), M, w.S5, Uf(sig), mu, sig, c7, g);
              nk += 2;
            }
          k_adj_in<<<grid2, 128, 0, cx.s>>>(w.G3, w.G5, Uf(rho), mu, rho, 1.0, g);
          k_adj_link<<<grid2, 128, 0, cx.s>>>(Df(rho), w.G5, w.S3, Uf(rho), mu, rho, 1.0, g);
          nk += 2;
        }
      }
      k_adj_in<<<grid2, 128, 0, cx.s>>>(Df(mu), w.G3, Uf(nu), mu, nu, 1.0, g);
      k_adj_link<<<grid2, 128, 0, cx.s>>>(Df(nu), w.G3, Uf(mu), Uf(nu), mu, nu, 1.0, g);
      nk += 2;
    }
  }
  if (midN && c[5] != 0)
    for (int mu = 0; mu < 4; mu++) {
      k_adj_naik<<<grid2, 128, 0, cx.s>>>(Df(mu), midN + mu * F1, Uf(mu), mu, c[5], g);
      nk++;
    }
  if (lepage_rep && cL != 0) {
    double2 *H[4] = {w.S3, w.S5, w.G3, w.G5};   // free once the sweep is done
    for (int nu = 0; nu < 4; nu++) k_lep_h<<<grid2, 128, 0, cx.s>>>(H[nu], mid + nu * F1, Uf(nu), nu, g);
    for (int mu = 0; mu < 4; mu++) {
      const double2 *o[3];
      for (int nu = 0, k = 0; nu < 4; nu++)
        if (nu != mu) o[k++] = H[nu];
      k_lep_fix<<<grid2, 128, 0, cx.s>>>(Df(mu), Uf(mu), o[0], o[1], o[2], mu, cL, g);
    }
    nk += 8;
  }
  QLAUNCHN(nk);
  return nk;
}

// outer products of sources [first, first + n) into mid (and midN)
template <typename T>
void force_mids(double2 *mid, double2 *midN, VecT<T> *const *x, const double *w, int n, double even_sign) {
  Context &cx = ctx();
  std::vector<const c2<T> *> hx(n);
  for (int k = 0; k < n; k++) hx[k] = x[k]->d;
  const c2<T> **dx = dalloc<const c2<T> *>(n);
  double *dw = dalloc<double>(n);
  QCHECK(cudaMemcpyAsync(dx, hx.data(), sizeof(void *) * n, cudaMemcpyHostToDevice, cx.s));
  QCHECK(cudaMemcpyAsync(dw, w, sizeof(double) * n, cudaMemcpyHostToDevice, cx.s));
  k_force_mid<T><<<grid_for(2 * cx.g.Vh, 128), 128, 0, cx.s>>>(mid, midN, dx, dw, n, even_sign, cx.g);
  QLAUNCH();
  dfree(dx);
  dfree(dw);
}

}  // namespace

template <typename T>
void asqtad_force(QOP_info_t *info, GaugeT<T> *G, GaugeT<T> *F, const QOP_asqtad_coeffs_t *cf, const double *eps,
                  VecT<T> *const *x, int nsrc) {
  Context &c = ctx();
  const Geom &g = c.g;
  const double t0 = wtime();
  const i64 Vh = g.Vh, F1 = 18 * Vh, F4 = 72 * Vh;
  bool own = false;
  double2 *U = gauge_fp64(G, own);
  const bool naik = cf->naik != 0;
  double2 *mid = dalloc<double2>(naik ? 2 * F4 : F4), *D = dalloc<double2>(F4);
  dzero(D, sizeof(double2) * F4);
  const SweepWork w{dalloc<double2>(F1), dalloc<double2>(F1), dalloc<double2>(F1), dalloc<double2>(F1)};
  force_mids<T>(mid, naik ? mid + F4 : nullptr, x, eps, nsrc, -1.0);   // scale -1 (fnmat_p.c:497)
  const double co[6] = {cf->one_link, cf->three_staple, cf->five_staple, cf->seven_staple, cf->lepage, cf->naik};
  const int nk = smear_adjoint(U, co, mid, naik ? mid + F4 : nullptr, D, w);
  // the reference's algorithm choice (lib/asqtad_force_p.c:22): FNMAT adds
  // -2 TA(U D^+); ASVEC (fewer sources than fnmat_src_min) stores
  // TA(force + C) with TA(C) = -TA(U D^+), half the FNMAT term
  const bool asvec = nsrc < c.opt.force_fnmat_src_min;
  if (asvec) {
    k_force_ta_self<T><<<grid_for(8 * Vh, 128), 128, 0, c.s>>>(F->d, g);
    QLAUNCH();
  }
  k_force_ta<T><<<grid_for(8 * Vh, 128), 128, 0, c.s>>>(F->d, U, D, asvec ? -1.0 : -2.0, g);
  QLAUNCH();
  sync();
  dfree(mid); dfree(D); dfree(w.S3); dfree(w.S5); dfree(w.G3); dfree(w.G5);
  if (own) dfree(U);
  if (info) {
    info->final_sec = wtime() - t0;
    // outer products, adjoint staples (~4 matrix products each) and projection
    info->final_flop = (double)g.V * (4.0 * (naik ? 2 : 1) * 72 * nsrc + nk * 216.0 + 4 * 264);
    info->status = QOP_SUCCESS;
  }
}

template <typename T>
void hisq_force(QOP_info_t *info, HisqT<T> *h, GaugeT<T> *F, const QOP_hisq_coeffs_t *cf, const double *res,
                VecT<T> *const *x, const int *n_orders) {
  Context &c = ctx();
  const Geom &g = c.g;
  const double t0 = wtime();
  if (!h->U || !h->V || !h->W)
    fail(QOP_FAIL, "hisq_force: the HISQ links carry no auxiliary U/V/W fields "
                   "(create them with QOP_hisq_links_set_opts want_aux = 1)");
  const i64 Vh = g.Vh, F1 = 18 * Vh, F4 = 72 * Vh;
  bool oU = false, oV = false, oW = false;
  double2 *U = gauge_fp64(h->U, oU), *V = gauge_fp64(h->V, oV), *W = gauge_fp64(h->W, oW);
  double2 *mid = dalloc<double2>(2 * F4), *GW = dalloc<double2>(F4), *T1 = dalloc<double2>(F4);
  double2 *D = dalloc<double2>(F4);
  dzero(GW, sizeof(double2) * F4);
  dzero(D, sizeof(double2) * F4);
  const SweepWork w{dalloc<double2>(F1), dalloc<double2>(F1), dalloc<double2>(F1), dalloc<double2>(F1)};
  int nterms = 0;
  for (int k = 0; k < cf->n_naiks; k++) nterms += n_orders[k];
  const double ca[6] = {cf->asqtad_one_link, cf->asqtad_three_staple, cf->asqtad_five_staple,
                        cf->asqtad_seven_staple, cf->asqtad_lepage, cf->asqtad_naik};
  const double cd[6] = {cf->difference_one_link, 0, 0, 0, 0, cf->difference_naik};
  int nk = 0, shift = 0;
  for (int k = 0; k < cf->n_naiks; k++) {
    // group 0 takes every source with the asqtad coefficients, group k >= 1
    // its own sources with the difference coefficients (fnmat2_p.c:52-113)
    const int first = k == 0 ? 0 : shift, count = k == 0 ? nterms : n_orders[k];
    shift += n_orders[k];
    if (count == 0) continue;
    force_mids<T>(mid, mid + F4, x + first, res + first, count, 1.0);
    dzero(T1, sizeof(double2) * F4);
    nk += smear_adjoint(W, k == 0 ? ca : cd, mid, mid + F4, T1, w, true);
    k_field_axpby<<<grid_for(F4, 256), 256, 0, c.s>>>(GW, 1.0, T1, k == 0 ? 1.0 : cf->eps_naik[k], F4);
    QLAUNCH();
  }
  k_reunit_adj<<<grid_for(8 * Vh, 128), 128, 0, c.s>>>(T1, V, GW, 8 * Vh, c.opt.hisq_force_filter);   // T1 = GV
  QLAUNCH();
  const double c7[6] = {cf->fat7_one_link, cf->fat7_three_staple, cf->fat7_five_staple, cf->fat7_seven_staple,
                        c.opt.use_fat7_lepage ? cf->fat7_lepage : 0.0, 0.0};
  nk += smear_adjoint(U, c7, T1, nullptr, D, w);
  k_force_ta<T><<<grid_for(8 * Vh, 128), 128, 0, c.s>>>(F->d, U, D, 2.0, g);   // deriv = 2 D
  QLAUNCH();
  sync();
  dfree(mid); dfree(GW); dfree(T1); dfree(D); dfree(w.S3); dfree(w.S5); dfree(w.G3); dfree(w.G5);
  if (oU) dfree(U);
  if (oV) dfree(V);
  if (oW) dfree(W);
  if (info) {
    info->final_sec = wtime() - t0;
    info->final_flop = (double)g.V * (8.0 * 72 * nterms + nk * 216.0 + 4 * 1500 + 4 * 264);
    info->status = QOP_SUCCESS;
  }
}

template void asqtad_force<float>(QOP_info_t *, GaugeT<float> *, GaugeT<float> *, const QOP_asqtad_coeffs_t *,
                                  const double *, VecT<float> *const *, int);
template void asqtad_force<double>(QOP_info_t *, GaugeT<double> *, GaugeT<double> *, const QOP_asqtad_coeffs_t *,
                                   const double *, VecT<double> *const *, int);
template void hisq_force<float>(QOP_info_t *, HisqT<float> *, GaugeT<float> *, const QOP_hisq_coeffs_t *,
                                const double *, VecT<float> *const *, const int *);
template void hisq_force<double>(QOP_info_t *, HisqT<double> *, GaugeT<double> *, const QOP_hisq_coeffs_t *,
                                 const double *, VecT<double> *const *, const int *);

}  // namespace qopb
