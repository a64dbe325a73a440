// bmma.cuh -- the tensor-core form of the batched hop (batch_kernel 16) and
// the vector format it works on.
//
// Per site and slot the batched hop is a 3x3 complex link times a 3 x n block
// of right-hand sides.  As a real product over all slots of a site:
//   C (16 systems x 8) = A (16 systems x 16 slots x 8) . B (16 slots x 8 x 8)
// A row j holds system j's neighbour sites (colour c, re / im in the k
// positions 8s + 2c, 8s + 2c + 1; k = 8s + 6, 8s + 7 are padding), B the
// slot's link in real form (output colour r, re / im in column 2r, 2r + 1;
// columns 6, 7 zero): one warp issues mma.sync.m16n8k16 (bf16 in, FP32
// accumulate) per pair of slots.  Precision: every FP32 operand x is split
// into bf16 hi = bf16(x) and lo = bf16(x - hi) (16 bits of mantissa
// together), and the product is hi.hi + hi.lo + lo.hi (three MMAs) with FP32
// accumulation: an FP32 product to ~2^-17, finer than the int16 storage (15
// bits) of the other sloppy formats.
//
// Vectors of the tensor-core batched solver are stored already split: a
// record per (site, system) of 24 bytes = 3 colours x {hi bf16x2 (re, im),
// lo bf16x2 (re, im)}, 16 systems per site, sites in checkerboard order
// ([Vh][16] records).  A lane of the MMA loads its A fragment straight from
// a record (one 8-byte load per colour: no decode), and the 16 systems of a
// neighbour site are 384 contiguous bytes.
#pragma once
#include "mixed.cuh"
#include <cuda_bf16.h>

namespace qopb {

constexpr int BSYS = 16;   // systems per site in the tensor-core format

struct B16Rec {
  uint2 c[3];   // per colour: x = hi (re low half, im high half), y = lo
};
static_assert(sizeof(B16Rec) == 24, "a record is 3 colours x 8 bytes");

// one FP32 complex value as its hi / lo bf16 pairs (re in the low half)
__device__ __forceinline__ uint2 b16_split(float re, float im) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(re, im);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(re - hf.x, im - hf.y);
  return make_uint2(*reinterpret_cast<const unsigned *>(&h), *reinterpret_cast<const unsigned *>(&l));
}
__device__ __forceinline__ float2 b16_join(uint2 v) {
  const float2 h = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&v.x));
  const float2 l = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&v.y));
  return make_float2(h.x + l.x, h.y + l.y);
}

// FP64 parity block [3][Vh] of system j <-> the tensor-core format
__global__ void k_b16_from_f64(B16Rec *v, int j, const double2 *src, i64 Vh);
__global__ void k_b16_to_f64(double2 *dst, const B16Rec *v, int j, i64 Vh);
__global__ void k_b16_copy_sys(B16Rec *dst, const B16Rec *src, int j, i64 Vh);
// xs: FP32 solution accumulators [Vh][16][3] float2
__global__ void k_b16_zero_x(float2 *xs, int j, i64 Vh);
__global__ void k_b16_fold_x(double2 *x, float2 *xs, int j, i64 Vh);   // x += xs_j, xs_j = 0

// t_j = D_oe p_j (kind 1, sums |t_j|^2 into dp2) or Ap_j = m_j^2 p_j - D_eo t_j
// (kind 2, sums |p_j|^2 and sets alpha_j) for the systems j < nsys whose
// state flag is clear; lk = the int16 links of the output parity (blocked,
// mixed.cuh); part holds bmma_part_doubles() doubles, count one ticket
void launch_bmma_hop(int kind, int nl, bool recon, float c_long, B16Rec *out, const B16Rec *src,
                     const unsigned char *lk, const B16Rec *same, const Geom &g, const NbrGeom &ng, int par,
                     MixState *st, int nsys, double *part, unsigned *count);
// x_j += alpha_j p_j, r_j -= alpha_j Ap_j, |r_j|^2 -> beta_j and the update
// test, for the running systems
void launch_b16_update(float2 *xs, B16Rec *r, const B16Rec *p, const B16Rec *Ap, i64 Vh, MixState *st, int nsys,
                       double *part, unsigned *count);
// p_j = r_j + beta_j p_j for the running systems (only system `only` if >= 0)
void launch_b16_p(B16Rec *p, const B16Rec *r, i64 Vh, const MixState *st, int nsys, int only = -1);
// partial sums the launchers above need (doubles)
size_t bmma_part_doubles();

}  // namespace qopb
