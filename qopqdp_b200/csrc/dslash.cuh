// dslash.cuh -- site geometry and the asqtad hop stencil shared by kernels.
#pragma once
#include "qopb.h"

namespace qopb {

// coordinates of checkerboard site i in parity p (inverse of layout_user.c
// :237-258 restricted to one parity; needs L[3] even)
__device__ __forceinline__ void site_coords(const Geom &g, int i, int p, int x[4]) {
  int l = 2 * i;
  int x3 = l % g.L[3];
  int q = l / g.L[3];
  x[2] = q % g.L[2];
  q /= g.L[2];
  x[1] = q % g.L[1];
  x[0] = q / g.L[1];
  x[3] = x3 + ((x[0] + x[1] + x[2] + x3 + p) & 1);
}

__device__ __forceinline__ int site_index(const Geom &g, int x0, int x1, int x2, int x3) {
  return (((x0 * g.L[1] + x1) * g.L[2] + x2) * g.L[3] + x3) >> 1;
}

// neighbour x + d*mu (|d| <= 3 < L) as a checkerboard index
__device__ __forceinline__ int nbr_index(const Geom &g, const int x[4], int mu, int d) {
  int y[4] = {x[0], x[1], x[2], x[3]};
  int t = y[mu] + d;
  int L = g.L[mu];
  t = t >= L ? t - L : (t < 0 ? t + L : t);
  y[mu] = t;
  return site_index(g, y[0], y[1], y[2], y[3]);
}

// slot k of the double-stored link set: direction and displacement
template <int NL> __device__ __forceinline__ int slot_mu(int k) { return NL == 16 ? (k >> 2) : (k >> 1); }
template <int NL> __device__ __forceinline__ int slot_disp(int k) {
  if (NL == 16) { int r = k & 3; return r == 0 ? 1 : r == 1 ? 3 : r == 2 ? -1 : -3; }
  return (k & 1) ? -1 : 1;
}
inline int host_slot_mu(int nl, int k) { return nl == 16 ? (k >> 2) : (k >> 1); }
inline int host_slot_disp(int nl, int k) {
  if (nl == 16) { int r = k & 3; return r == 0 ? 1 : r == 1 ? 3 : r == 2 ? -1 : -3; }
  return (k & 1) ? -1 : 1;
}

}  // namespace qopb
