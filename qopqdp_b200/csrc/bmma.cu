// bmma.cu -- tensor-core batched hop (mma.sync.m16n8k16, bf16 hi/lo split
// operands, FP32 accumulation) and the elementwise kernels of the batched
// solver in the tensor-core vector format (bmma.cuh).  Reference: the hop
// over nsvec vectors of lib/asqtad_dslash_p.c:1212-1215,1246-1279 and the
// multi-source solves of lib/asqtad_invert_p.c:853-1059.
//
// Hop kernel, one block of 8 warps per chunk of 32 sites (persistent grid,
// two blocks per SM):
//  0. the block computes the coordinates of the chunk's sites once and the
//     neighbour index of every (site, slot) into shared memory;
//  1. it decodes the int16 links of the chunk (every link once) into
//     shared memory as B fragments: for (site, slot) the 18 lanes (g < 6,
//     q < 3) that carry link data get link element (g/2, q) as (re, -im)
//     for even g and (im, re) for odd g, each split into bf16 hi / lo pairs
//     (8 bytes per lane; the even / odd words of an element are adjacent and
//     written by one 16-byte store);
//  2. each warp takes 4 sites; per site every lane requests its A fragments
//     for all 16 slots at once (the hi / lo words of colour q of systems g
//     and g + 8 at each neighbour: two 8-byte loads per slot, no decode),
//     then per pair of slots loads its B fragment from shared memory and
//     issues three MMAs (hi.hi, hi.lo, lo.hi) into three accumulator sets;
//     lane (g, q < 3) ends with colour q of the output of systems g, g + 8;
//  3. epilogue per site: kind 1 stores t = D p (split) and sums |t|^2; kind 2
//     combines with p at the site (requested with the fragments), stores
//     Ap = m^2 p - t and sums |p|^2; the per-system sums go through a
//     deterministic grid reduction whose last block sets dp2 or alpha of
//     every running system.
#include "bmma.cuh"
#include "dslash.cuh"
#include "reduce.cuh"
#include <cuda_bf16.h>
#include <mutex>

namespace qopb {

constexpr int BM_SITES = 32;        // sites per chunk
constexpr int BM_THREADS = 256;     // 8 warps
constexpr int BM_LW = 18;           // B-fragment lanes that carry link data (g < 6, q < 3)
// words (8 bytes) per site in the fragment table: NL x 18, plus two so that
// the threads decoding consecutive sites of one slot store to different
// banks (a stride of 2304 bytes would put them all on one; measured: 127
// conflicts per site) and every 16-byte store stays aligned.  Within a
// (site, slot) the word of lane (g, q) is q x 6 + g.
template <int NL> constexpr int bm_site_words() { return NL * BM_LW + 2; }

// not volatile: the MMA has no side effects, so the compiler may schedule
// the operand loads freely around it
__device__ __forceinline__ void mma_bf16(float (&c)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                         unsigned b0, unsigned b1) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// the int16 link decodes of the batched hop (batch.cu), for the fragments:
// integer-valued elements and the factor that scales them
__device__ __forceinline__ float bm_link(const uint4 ua, const uint4 ub, const uint2 uc, float2 U[9]) {
  U[0] = u16_pair(ua.x); U[1] = u16_pair(ua.y); U[2] = u16_pair(ua.z); U[3] = u16_pair(ua.w);
  U[4] = u16_pair(ub.x); U[5] = u16_pair(ub.y); U[6] = u16_pair(ub.z); U[7] = u16_pair(ub.w);
  U[8] = u16_pair(uc.x);
  return __uint_as_float(uc.y) * (1.0f / 32767.0f);
}
__device__ __forceinline__ float bm_link_recon(const uint4 ua, const uint2 ub, const float phase, const float cl,
                                               float2 U[9]) {
  U[0] = u16_pair(ua.x); U[1] = u16_pair(ua.y); U[2] = u16_pair(ua.z); U[3] = u16_pair(ua.w);
  U[4] = u16_pair(ub.x); U[5] = u16_pair(ub.y);
  float sn, cs;
  __sincosf(phase, &sn, &cs);
  const float2 z = make_float2(cs * (1.0f / 32767.0f), sn * (1.0f / 32767.0f));
  const float2 c0 = csub<float>(cmul<float>(U[1], U[5]), cmul<float>(U[2], U[4]));
  const float2 c1 = csub<float>(cmul<float>(U[2], U[3]), cmul<float>(U[0], U[5]));
  const float2 c2 = csub<float>(cmul<float>(U[0], U[4]), cmul<float>(U[1], U[3]));
  U[6] = cmul<float>(z, make_float2(c0.x, -c0.y));
  U[7] = cmul<float>(z, make_float2(c1.x, -c1.y));
  U[8] = cmul<float>(z, make_float2(c2.x, -c2.y));
  return cl * (1.0f / 32767.0f);
}

template <int NL, int KIND, bool RECON>
__global__ void __launch_bounds__(BM_THREADS, 2)
k_bmma_hop(B16Rec *__restrict__ out, const B16Rec *__restrict__ src, const unsigned char *__restrict__ lk,
           const B16Rec *__restrict__ same, Geom g, NbrGeom ng, int p, MixState *st, int nsys, double *part,
           unsigned *count, float c_long) {
  extern __shared__ __align__(16) uint2 bfrag[];   // [BM_SITES][NL x BM_LW + 2]
  __shared__ double red[BM_THREADS / 32][BSYS];
  __shared__ int sx[BM_SITES][5];                   // coordinates and lex index of the chunk's sites
  __shared__ __align__(16) int snb[BM_SITES][NL];   // their neighbour indices per slot
  __shared__ bool am_last;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, qq = lane & 3;
  const i64 Vh = g.Vh;
  const int j0 = gq, j1 = gq + 8;
  const bool act0 = j0 < nsys && st[j0].flag == 0;
  const bool act1 = j1 < nsys && st[j1].flag == 0;
  // the flags are the same for every block: a launch with no running system
  // returns everywhere (no block reduces)
  if (!__any_sync(0xffffffffu, act0 || act1)) return;
  const float m2_0 = act0 ? (float)st[j0].m2 : 0.f, m2_1 = act1 ? (float)st[j1].m2 : 0.f;
  const bool lb = gq < 6 && qq < 3;
  // this lane's 8-byte word in a neighbour's record block: system g, colour
  // q.  Lanes q = 3 fill the padding columns k = 6, 7 of A with colour 2 of
  // their system (finite for a running system) instead of zero: B's rows
  // 6, 7 are zero, so those products add exactly 0.  Systems that are not
  // running load nothing (late in a multi-mass solve most have finished):
  // their A rows are zero, and an MMA row affects only the same row of C.
  const int lane_w = gq * 3 + (qq < 3 ? qq : 2);
  double acc0 = 0.0, acc1 = 0.0;
  const int nchunk = (int)((Vh + BM_SITES - 1) / BM_SITES);
  for (int ch = blockIdx.x; ch < nchunk; ch += gridDim.x) {
    const i64 base = (i64)ch * BM_SITES;
    __syncthreads();   // the previous chunk's tables are consumed
    // ---- 0. coordinates of the chunk's sites, then the neighbour index of
    // every (site, slot)
    if (tid < BM_SITES) {
      const i64 i = base + tid;
      int x[4] = {0, 0, 0, 0};
      if (i < Vh) site_coords(g, (int)i, p, x);
      sx[tid][0] = x[0]; sx[tid][1] = x[1]; sx[tid][2] = x[2]; sx[tid][3] = x[3];
      sx[tid][4] = ((x[0] * g.L[1] + x[1]) * g.L[2] + x[2]) * g.L[3] + x[3];
    }
    __syncthreads();
    for (int it = tid; it < BM_SITES * NL; it += BM_THREADS) {
      const int sl = it % BM_SITES, k = it / BM_SITES;
      snb[sl][k] = nbr_sel(ng, sx[sl][0], sx[sl][1], sx[sl][2], sx[sl][3], sx[sl][4], slot_mu<NL>(k), slot_disp<NL>(k));
    }
    // ---- 1. link fragments of the chunk: item = slot x 32 + site, so that
    // consecutive threads read consecutive sites of one slot (coalesced)
    for (int it = tid; it < BM_SITES * NL; it += BM_THREADS) {
      const int sl = it % BM_SITES, k = it / BM_SITES;
      const i64 i = base + sl;
      uint2 *dst = bfrag + sl * bm_site_words<NL>() + k * BM_LW;
      if (i >= Vh) {
#pragma unroll
        for (int e = 0; e < BM_LW; e += 2) *reinterpret_cast<uint4 *>(dst + e) = make_uint4(0u, 0u, 0u, 0u);
        continue;
      }
      const int t = (int)(i % QB);
      const unsigned char *ls = lk + (size_t)(i / QB) * q16_block_bytes(NL, RECON) + q16_slot_off(k, RECON);
      float2 U[9];
      float sc;
      if (RECON && (k & 1)) {
        const uint4 ua = __ldg(reinterpret_cast<const uint4 *>(ls) + t);
        const uint2 ub = __ldg(reinterpret_cast<const uint2 *>(ls + 16 * QB) + t);
        const float ph = __ldg(reinterpret_cast<const float *>(ls + 24 * QB) + t);
        sc = bm_link_recon(ua, ub, ph, c_long, U);
      } else {
        const uint4 ua = __ldg(reinterpret_cast<const uint4 *>(ls) + t);
        const uint4 ub = __ldg(reinterpret_cast<const uint4 *>(ls + 16 * QB) + t);
        const uint2 uc = __ldg(reinterpret_cast<const uint2 *>(ls + 32 * QB) + t);
        sc = bm_link(ua, ub, uc, U);
      }
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const uint2 s = b16_split(U[3 * r + c].x * sc, U[3 * r + c].y * sc);
          // even g = 2r: (re, -im); odd g = 2r + 1: (im, re); one 16-byte store
          *reinterpret_cast<uint4 *>(dst + c * 6 + 2 * r) =
              make_uint4(s.x ^ 0x80000000u, s.y ^ 0x80000000u, __byte_perm(s.x, 0u, 0x1032),
                         __byte_perm(s.y, 0u, 0x1032));
        }
    }
    __syncthreads();
    // ---- 2. four sites per warp
    for (int sl = warp; sl < BM_SITES; sl += BM_THREADS / 32) {
      const i64 i = base + sl;
      if (i >= Vh) break;   // warp-uniform; the later sites of the chunk are past Vh too
      // every A fragment of the site is requested before the first MMA, so
      // the 2 NL loads of a lane are in flight together
      uint2 ra[NL][2];
#pragma unroll
      for (int s = 0; s < NL; s += 4) {
        const int4 n4 = *reinterpret_cast<const int4 *>(&snb[sl][s]);
        const int nn[4] = {n4.x, n4.y, n4.z, n4.w};
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const uint2 *ap = reinterpret_cast<const uint2 *>(src + (i64)nn[u] * BSYS) + lane_w;
          ra[s + u][0] = act0 ? __ldg(ap) : make_uint2(0u, 0u);
          ra[s + u][1] = act1 ? __ldg(ap + 24) : make_uint2(0u, 0u);
        }
      }
      // kind 2: p at the output site, requested with the fragments
      uint2 pw0 = make_uint2(0u, 0u), pw1 = pw0;
      if (KIND == 2 && qq < 3) {
        if (act0) pw0 = __ldg(&same[i * BSYS + j0].c[qq]);
        if (act1) pw1 = __ldg(&same[i * BSYS + j1].c[qq]);
      }
      // three accumulator sets (hi.hi, hi.lo, lo.hi): three independent
      // chains of NL / 2 MMAs instead of one of 3 NL / 2
      float c[4] = {0.f, 0.f, 0.f, 0.f}, cl[4] = {0.f, 0.f, 0.f, 0.f}, chh[4] = {0.f, 0.f, 0.f, 0.f};
      const uint2 *bf = bfrag + sl * bm_site_words<NL>() + qq * 6 + gq;
#pragma unroll
      for (int s = 0; s < NL; s += 2) {
        uint2 b0 = make_uint2(0u, 0u), b1 = b0;
        if (lb) {
          b0 = bf[s * BM_LW];
          b1 = bf[(s + 1) * BM_LW];
        }
        const uint2 r0 = ra[s][0], r1 = ra[s][1], r2 = ra[s + 1][0], r3 = ra[s + 1][1];
        mma_bf16(c, r0.x, r1.x, r2.x, r3.x, b0.x, b1.x);     // hi . hi
        mma_bf16(cl, r0.x, r1.x, r2.x, r3.x, b0.y, b1.y);    // hi . lo
        mma_bf16(chh, r0.y, r1.y, r2.y, r3.y, b0.x, b1.x);   // lo . hi
      }
#pragma unroll
      for (int e = 0; e < 4; e++) c[e] += cl[e] + chh[e];
      // ---- 3. epilogue: lane (g, q < 3) holds colour q of systems g, g + 8
      if (qq < 3) {
        const i64 o0 = i * BSYS + j0, o1 = i * BSYS + j1;
        if (KIND == 1) {
          if (act0) {
            out[o0].c[qq] = b16_split(c[0], c[1]);
            acc0 += (double)c[0] * c[0] + (double)c[1] * c[1];
          }
          if (act1) {
            out[o1].c[qq] = b16_split(c[2], c[3]);
            acc1 += (double)c[2] * c[2] + (double)c[3] * c[3];
          }
        } else {
          if (act0) {
            const float2 pv = b16_join(pw0);
            out[o0].c[qq] = b16_split(m2_0 * pv.x - c[0], m2_0 * pv.y - c[1]);
            acc0 += (double)pv.x * pv.x + (double)pv.y * pv.y;
          }
          if (act1) {
            const float2 pv = b16_join(pw1);
            out[o1].c[qq] = b16_split(m2_1 * pv.x - c[2], m2_1 * pv.y - c[3]);
            acc1 += (double)pv.x * pv.x + (double)pv.y * pv.y;
          }
        }
      }
    }
  }
  // ---- per-system sums: lanes of a quad, warps, blocks (fixed order)
  acc0 += __shfl_xor_sync(0xffffffffu, acc0, 1);
  acc0 += __shfl_xor_sync(0xffffffffu, acc0, 2);
  acc1 += __shfl_xor_sync(0xffffffffu, acc1, 1);
  acc1 += __shfl_xor_sync(0xffffffffu, acc1, 2);
  if (qq == 0) {
    red[warp][j0] = acc0;
    red[warp][j1] = acc1;
  }
  __syncthreads();
  if (tid < BSYS) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < BM_THREADS / 32; w++) s += red[w][tid];
    part[(size_t)blockIdx.x * BSYS + tid] = s;
    __threadfence();
  }
  __syncthreads();
  if (tid == 0) am_last = atomicAdd(count, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  if (tid < nsys) {
    double s = 0.0;
    for (int b = 0; b < (int)gridDim.x; b++) s += __ldcg(part + (size_t)b * BSYS + tid);
    MixState *S = st + tid;
    if (S->flag == 0) {
      if (KIND == 1) {
        S->dp2 = s;
      } else {
        const double pAp = S->dp2 + S->m2 * s;   // <p, A p> = |D p|^2 + m^2 |p|^2
        if (!(pAp > 0)) S->flag = MIX_BREAK;
        else S->alpha = S->rsq / pAp;
      }
    }
  }
  if (tid == 0) *count = 0u;
}

// ---------------------------------------------------------------- elementwise kernels
__global__ void k_b16_from_f64(B16Rec *v, int j, const double2 *src, i64 Vh) {
  const i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (i >= Vh) return;
  B16Rec r;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const double2 w = src[c * Vh + i];
    r.c[c] = b16_split((float)w.x, (float)w.y);
  }
  v[i * BSYS + j] = r;
}

__global__ void k_b16_to_f64(double2 *dst, const B16Rec *v, int j, i64 Vh) {
  const i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (i >= Vh) return;
  const B16Rec r = v[i * BSYS + j];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float2 f = b16_join(r.c[c]);
    dst[c * Vh + i] = make_double2(f.x, f.y);
  }
}

__global__ void k_b16_copy_sys(B16Rec *dst, const B16Rec *src, int j, i64 Vh) {
  const i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (i < Vh) dst[i * BSYS + j] = src[i * BSYS + j];
}

__global__ void k_b16_zero_x(float2 *xs, int j, i64 Vh) {
  const i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (i >= Vh) return;
#pragma unroll
  for (int c = 0; c < 3; c++) xs[(i * BSYS + j) * 3 + c] = make_float2(0.f, 0.f);
}

__global__ void k_b16_fold_x(double2 *x, float2 *xs, int j, i64 Vh) {
  const i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (i >= Vh) return;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    float2 &s = xs[(i * BSYS + j) * 3 + c];
    double2 d = x[c * Vh + i];
    d.x += s.x;
    d.y += s.y;
    x[c * Vh + i] = d;
    s = make_float2(0.f, 0.f);
  }
}

// x_j += alpha_j p_j, r_j -= alpha_j Ap_j, |r_j|^2: one thread per (site,
// system), the system fixed per thread (blocks and strides are multiples of
// 16 records); the last block updates beta_j and the state of every system
constexpr int BU_THREADS = 256;
__global__ void __launch_bounds__(BU_THREADS)
k_b16_update(float2 *__restrict__ xs, B16Rec *__restrict__ r, const B16Rec *__restrict__ p,
             const B16Rec *__restrict__ Ap, i64 Vh, MixState *st, int nsys, double *part, unsigned *count) {
  __shared__ double red[BU_THREADS / 32][BSYS];
  __shared__ bool am_last;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int j = tid & (BSYS - 1);
  const bool act = j < nsys && st[j].flag == 0;
  double acc = 0.0;
  if (act) {
    const float al = (float)st[j].alpha;
    for (i64 e = blockIdx.x * (i64)BU_THREADS + tid; e < Vh * BSYS; e += (i64)gridDim.x * BU_THREADS) {
      const B16Rec pv = p[e], av = Ap[e];
      B16Rec rv = r[e];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const float2 pp = b16_join(pv.c[c]), aa = b16_join(av.c[c]);
        float2 rr = b16_join(rv.c[c]);
        float2 xv = xs[e * 3 + c];
        xv.x = fmaf(al, pp.x, xv.x);
        xv.y = fmaf(al, pp.y, xv.y);
        xs[e * 3 + c] = xv;
        rr.x = fmaf(-al, aa.x, rr.x);
        rr.y = fmaf(-al, aa.y, rr.y);
        rv.c[c] = b16_split(rr.x, rr.y);
        acc += (double)rr.x * rr.x + (double)rr.y * rr.y;
      }
      r[e] = rv;
    }
  }
  acc += __shfl_xor_sync(0xffffffffu, acc, 16);
  if (lane < BSYS) red[warp][lane] = acc;
  __syncthreads();
  if (tid < BSYS) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < BU_THREADS / 32; w++) s += red[w][tid];
    part[(size_t)blockIdx.x * BSYS + tid] = s;
    __threadfence();
  }
  __syncthreads();
  if (tid == 0) am_last = atomicAdd(count, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  if (tid < nsys) {
    MixState *s = st + tid;
    if (s->flag == 0) {
      double rn = 0.0;
      for (int b = 0; b < (int)gridDim.x; b++) rn += __ldcg(part + (size_t)b * BSYS + tid);
      s->iter += 1;
      s->rsq_old = s->rsq;
      s->rsq = rn;
      s->beta = rn / s->rsq_old;
      if (rn > s->maxr2) s->maxr2 = rn;
      if (rn < s->delta2 * s->maxr2 || rn <= s->stop || s->iter >= s->max_iter) s->flag = MIX_UPDATE;
    }
  }
  if (tid == 0) *count = 0u;
}

// p_j = r_j + beta_j p_j for the running systems (or for system `only`)
__global__ void __launch_bounds__(BU_THREADS)
k_b16_p(B16Rec *__restrict__ p, const B16Rec *__restrict__ r, i64 Vh, const MixState *st, int nsys, int only) {
  const i64 n = only >= 0 ? Vh : Vh * BSYS;
  for (i64 e0 = blockIdx.x * (i64)BU_THREADS + threadIdx.x; e0 < n; e0 += (i64)gridDim.x * BU_THREADS) {
    const i64 e = only >= 0 ? e0 * BSYS + only : e0;
    const int j = (int)(e & (BSYS - 1));
    if (j >= nsys || st[j].flag) continue;
    const float be = (float)st[j].beta;
    const B16Rec rv = r[e];
    B16Rec pv = p[e];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float2 pp = b16_join(pv.c[c]), rr = b16_join(rv.c[c]);
      pv.c[c] = b16_split(fmaf(be, pp.x, rr.x), fmaf(be, pp.y, rr.y));
    }
    p[e] = pv;
  }
}

// ---------------------------------------------------------------- launchers
namespace {
int update_grid(i64 Vh) {
  const i64 b = (Vh * BSYS + BU_THREADS - 1) / BU_THREADS;
  return (int)std::max<i64>(1, std::min<i64>(b, (i64)ctx().red_blocks * 2));
}

struct HopCfg {
  int grid = 0;
  size_t smem = 0;
};

template <int NL, int KIND, bool RECON>
HopCfg hop_cfg() {
  static HopCfg cfg;
  static std::once_flag once;
  std::call_once(once, [] {
    auto k = k_bmma_hop<NL, KIND, RECON>;
    cfg.smem = (size_t)BM_SITES * bm_site_words<NL>() * sizeof(uint2);
    QCHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem));
    int occ = 0;
    QCHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, BM_THREADS, cfg.smem));
    int sms = 0;
    QCHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx().device));
    cfg.grid = std::max(1, occ) * sms;
  });
  return cfg;
}

template <int NL, int KIND, bool RECON>
void launch_t(float c_long, B16Rec *out, const B16Rec *src, const unsigned char *lk, const B16Rec *same,
              const Geom &g, const NbrGeom &ng, int par, MixState *st, int nsys, double *part, unsigned *count) {
  const HopCfg cfg = hop_cfg<NL, KIND, RECON>();
  const int nchunk = (int)((g.Vh + BM_SITES - 1) / BM_SITES);
  const int grid = std::min(cfg.grid, nchunk);
  k_bmma_hop<NL, KIND, RECON><<<grid, BM_THREADS, cfg.smem, ctx().s>>>(out, src, lk, same, g, ng, par, st, nsys,
                                                                       part, count, c_long);
}
}  // namespace

size_t bmma_part_doubles() {
  int sms = 0;
  QCHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx().device));
  // hop grids are SMs x (resident blocks <= 8); update grids <= 2 red_blocks
  return (size_t)BSYS * std::max<size_t>((size_t)sms * 8, (size_t)ctx().red_blocks * 2);
}

void launch_bmma_hop(int kind, int nl, bool recon, float c_long, B16Rec *out, const B16Rec *src,
                     const unsigned char *lk, const B16Rec *same, const Geom &g, const NbrGeom &ng, int par,
                     MixState *st, int nsys, double *part, unsigned *count) {
#define BM_ARGS c_long, out, src, lk, same, g, ng, par, st, nsys, part, count
  if (nl != 16) {
    if (kind == 1) launch_t<8, 1, false>(BM_ARGS);
    else launch_t<8, 2, false>(BM_ARGS);
  } else if (recon) {
    if (kind == 1) launch_t<16, 1, true>(BM_ARGS);
    else launch_t<16, 2, true>(BM_ARGS);
  } else {
    if (kind == 1) launch_t<16, 1, false>(BM_ARGS);
    else launch_t<16, 2, false>(BM_ARGS);
  }
#undef BM_ARGS
}

void launch_b16_update(float2 *xs, B16Rec *r, const B16Rec *p, const B16Rec *Ap, i64 Vh, MixState *st, int nsys,
                       double *part, unsigned *count) {
  k_b16_update<<<update_grid(Vh), BU_THREADS, 0, ctx().s>>>(xs, r, p, Ap, Vh, st, nsys, part, count);
}

void launch_b16_p(B16Rec *p, const B16Rec *r, i64 Vh, const MixState *st, int nsys, int only) {
  const i64 n = only >= 0 ? Vh : Vh * BSYS;
  const int grid =
      (int)std::max<i64>(1, std::min<i64>((n + BU_THREADS - 1) / BU_THREADS, (i64)ctx().red_blocks * 4));
  k_b16_p<<<grid, BU_THREADS, 0, ctx().s>>>(p, r, Vh, st, nsys, only);
}

}  // namespace qopb
