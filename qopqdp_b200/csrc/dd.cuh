// dd.cuh -- halos of a decomposed lattice for the hop kernels (dd.cu).
//
// Each process holds a block of the global lattice with even local extents
// at an even global origin, so a local site's parity is its global parity
// and the node-local raw order is the single-lattice raw order of the block
// (lib/layout_user.c:238-258 with even blocks).  A hop from an output site
// x leaves the block along a decomposed direction mu when x_mu + d is < 0 or
// >= L_mu; the term then comes from a halo received before the hop:
//   up[mu]: the input vector at the sites x_mu = L_mu + j (j < depth) of the
//           +mu neighbour, multiplied by the local forward link as usual;
//   dn[mu]: -U_mu(y)^+ psi(y) at the sites y of the -mu neighbour, formed by
//           the neighbour with its own forward links (slab 0: fat link at
//           y_mu = -1; slab 1 + j: long link at y_mu = -1 - j), added as is.
// So the backward links of the boundary sites never leave their owner and
// no link halos exist.  Halo element (slab s, colour c, face site f) sits
// at [(s * 3 + c) * fh + f], f = floor(lex'/2) with lex' the lexicographic
// index of the three other coordinates (x0 slowest).  Every local extent is
// even, so lex' and lex'+1 of one pair have opposite parities and f is a
// bijection onto one parity's face sites.
#pragma once
#include "qopb.h"

namespace qopb {

template <typename T> struct DdGhost {
  const c2<T> *up[4];
  const c2<T> *dn[4];
  int fh[4];    // sites of one parity in one face slab of direction mu
  int mask;     // decomposed directions (bit mu)
};

// halo slabs: depth of the raw halo and number of product slabs
__host__ __device__ inline int dd_depth(int nl) { return nl == 16 ? 3 : 1; }
__host__ __device__ inline int dd_nprod(int nl) { return nl == 16 ? 4 : 1; }

// The halo plan.  These index functions are the only place the layout of
// the halos is defined: the pack kernels (producer), the hop kernels
// (consumer) and the host-side test hooks QOPB_dd_pack_site /
// QOPB_dd_halo_ref all call them.

// face index of local site x in a slab of direction mu
__host__ __device__ inline int dd_face_index_L(const int L[4], const int x[4], int mu) {
  int l = 0;
#pragma unroll
  for (int nu = 0; nu < 4; nu++)
    if (nu != mu) l = l * L[nu] + x[nu];
  return l >> 1;
}
__device__ __forceinline__ int dd_face_index(const Geom &g, const int x[4], int mu) {
  return dd_face_index_L(g.L, x, mu);
}

// consumer: a hop term (mu, d) from local site x leaves the block when
// y = x_mu + d is outside [0, L_mu); it reads up-halo slab y - L_mu, or
// down-halo slab 0 (the fat product, d = -1) or -y (the long products)
__host__ __device__ inline int dd_halo_slab(int Lmu, int y, int d) {
  return y < 0 ? (d == -1 ? 0 : -y) : y - Lmu;
}

// producer: the local site packed at (slab s, face index fi) of direction
// mu for the parity-q input; returns the link slot multiplied into a
// product slab (s >= depth), or -1 for a raw slab (s < depth: x_mu = s, for
// the -mu neighbour's up halo).  Product slab depth + j holds -U^+ psi at
// x_mu = L_mu - 1 - max(j - 1, 0) with the fat link (j = 0) or the long
// link (j >= 1), for the +mu neighbour's down halo.
__host__ __device__ inline int dd_pack_site(const int L[4], int mu, int nl, int q, int s, int fi, int x[4]) {
  const int depth = dd_depth(nl);
  int xm, slot = -1;
  if (s < depth) {
    xm = s;
  } else {
    const int j = s - depth;
    xm = L[mu] - 1 - (j == 0 ? 0 : j - 1);
    slot = nl == 16 ? (j == 0 ? 4 * mu : 4 * mu + 1) : 2 * mu;
  }
  int rem = 2 * fi;
  for (int nu = 3; nu >= 0; nu--)
    if (nu != mu) { x[nu] = rem % L[nu]; rem /= L[nu]; }
  x[mu] = xm;
  if (((x[0] + x[1] + x[2] + x[3]) & 1) != q) x[mu == 3 ? 2 : 3] += 1;   // the pair's other site
  return slot;
}

// packs the input halo of parity q (in: the parity-q block [colour][Vh]) and
// exchanges it with the neighbours; returns the halos for the hop kernels
template <typename T> DdGhost<T> dd_halo(FlaT<T> *f, const c2<T> *in, int q);

// the same for the int16 sloppy solver: in holds the parity-q int16 site
// records (16 bytes each); the up halo carries records, the down halo the
// products -U^+ psi, formed with lq, the solver's blocked int16 links of
// parity q (nl slots, long links reconstructed with |c| = c_long when
// recon), and stored as int16 records
struct DdQ16Ghost {
  const uint4 *up[4];
  const uint4 *dn[4];
  int fh[4];
  int mask;
};
DdQ16Ghost dd_halo_q16(int nl, const unsigned char *lq, bool recon, float c_long, const uint4 *in, int q);

}  // namespace qopb
