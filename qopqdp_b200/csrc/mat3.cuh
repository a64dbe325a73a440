// mat3.cuh -- FP64 3x3 complex matrix algebra and matrix-field accessors
// shared by link smearing (links.cu) and the fermion force (force.cu).
// A matrix field is [2 parities][9 elements][Vh sites] double2.
#pragma once
#include "qopb.h"
#include "dslash.cuh"

namespace qopb {

// ---------------------------------------------------------------- 3x3 algebra
struct M3 { double2 e[9]; };

__device__ __forceinline__ M3 ld3(const double2 *base, i64 Vh) {
  M3 m;
#pragma unroll
  for (int k = 0; k < 9; k++) m.e[k] = base[k * Vh];
  return m;
}
__device__ __forceinline__ void st3(double2 *base, i64 Vh, const M3 &m) {
#pragma unroll
  for (int k = 0; k < 9; k++) base[k * Vh] = m.e[k];
}
__device__ __forceinline__ M3 mul(const M3 &a, const M3 &b) {   // a b
  M3 r;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      double2 s = make_double2(0, 0);
#pragma unroll
      for (int k = 0; k < 3; k++) cfma<double>(s, a.e[3 * i + k], b.e[3 * k + j]);
      r.e[3 * i + j] = s;
    }
  return r;
}
__device__ __forceinline__ M3 mul_na(const M3 &a, const M3 &b) {   // a b^+
  M3 r;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      double2 s = make_double2(0, 0);
#pragma unroll
      for (int k = 0; k < 3; k++) {
        double2 x = a.e[3 * i + k], y = b.e[3 * j + k];
        s.x += x.x * y.x + x.y * y.y;
        s.y += x.y * y.x - x.x * y.y;
      }
      r.e[3 * i + j] = s;
    }
  return r;
}
__device__ __forceinline__ M3 mul_an(const M3 &a, const M3 &b) {   // a^+ b
  M3 r;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      double2 s = make_double2(0, 0);
#pragma unroll
      for (int k = 0; k < 3; k++) {
        double2 x = a.e[3 * k + i], y = b.e[3 * k + j];
        s.x += x.x * y.x + x.y * y.y;
        s.y += x.x * y.y - x.y * y.x;
      }
      r.e[3 * i + j] = s;
    }
  return r;
}

// field accessors: a matrix field is [2][9][Vh]
__device__ __forceinline__ const double2 *fptr(const double2 *f, const Geom &g, int p, int i) {
  return f + (i64)p * 9 * g.Vh + i;
}

// site (p,i) -> coords; neighbour parity flips for odd displacement
__device__ __forceinline__ void shifted(const Geom &g, const int x[4], int mu, int d, int y[4]) {
  for (int k = 0; k < 4; k++) y[k] = x[k];
  int L = g.L[mu];
  int t = (y[mu] + d) % L;
  y[mu] = t < 0 ? t + L : t;
}
__device__ __forceinline__ void par_idx(const Geom &g, const int y[4], int &p, int &i) {
  p = (y[0] + y[1] + y[2] + y[3]) & 1;
  i = site_index(g, y[0], y[1], y[2], y[3]);
}

// Hermitian Jacobi diagonalisation Q = Z diag(w) Z^+ (SVD stand-in)
static __device__ void herm_eig3(const M3 &Qin, double w[3], M3 &Z) {
  M3 A = Qin;
  for (int k = 0; k < 9; k++) Z.e[k] = make_double2(k % 4 == 0 ? 1.0 : 0.0, 0.0);
  for (int sweep = 0; sweep < 60; sweep++) {
    double off = 0;
    for (int p = 0; p < 3; p++)
      for (int q = p + 1; q < 3; q++) off += A.e[3 * p + q].x * A.e[3 * p + q].x + A.e[3 * p + q].y * A.e[3 * p + q].y;
    if (off < 1e-34) break;
    for (int p = 0; p < 3; p++)
      for (int q = p + 1; q < 3; q++) {
        double2 apq = A.e[3 * p + q];
        double r = hypot(apq.x, apq.y);
        if (r < 1e-300) continue;
        double app = A.e[4 * p].x, aqq = A.e[4 * q].x;
        double2 ph = make_double2(apq.x / r, apq.y / r);
        double theta = 0.5 * atan2(2 * r, aqq - app);
        double c = cos(theta), s = sin(theta);
        double2 gpp = make_double2(c, 0), gpq = make_double2(s * ph.x, s * ph.y);
        double2 gqp = make_double2(-s * ph.x, s * ph.y), gqq = make_double2(c, 0);
        for (int k = 0; k < 3; k++) {
          double2 akp = A.e[3 * k + p], akq = A.e[3 * k + q];
          A.e[3 * k + p] = cadd<double>(cmul<double>(akp, gpp), cmul<double>(akq, gqp));
          A.e[3 * k + q] = cadd<double>(cmul<double>(akp, gpq), cmul<double>(akq, gqq));
          double2 zkp = Z.e[3 * k + p], zkq = Z.e[3 * k + q];
          Z.e[3 * k + p] = cadd<double>(cmul<double>(zkp, gpp), cmul<double>(zkq, gqp));
          Z.e[3 * k + q] = cadd<double>(cmul<double>(zkp, gpq), cmul<double>(zkq, gqq));
        }
        for (int k = 0; k < 3; k++) {
          double2 apk = A.e[3 * p + k], aqk = A.e[3 * q + k];
          A.e[3 * p + k] = cadd<double>(cconjmul<double>(gpp, apk), cconjmul<double>(gqp, aqk));
          A.e[3 * q + k] = cadd<double>(cconjmul<double>(gpq, apk), cconjmul<double>(gqq, aqk));
        }
      }
  }
  for (int i = 0; i < 3; i++) w[i] = A.e[4 * i].x;
}

// FP64 copy of a gauge field ([4][2][9][Vh]); `owned` tells the caller to
// free it (links.cu)
template <typename T> double2 *gauge_fp64(GaugeT<T> *G, bool &owned);

}  // namespace qopb
