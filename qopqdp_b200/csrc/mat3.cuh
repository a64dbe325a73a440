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

// FP64 copy of a gauge field ([4][2][9][Vh]); `owned` tells the caller to
// free it (links.cu)
template <typename T> double2 *gauge_fp64(GaugeT<T> *G, bool &owned);

}  // namespace qopb
