// batch.cu -- several independent systems A_j x_j = b_j, A_j = m_j^2 - D_eo D_oe
// on one parity, solved together (B200 addition; the reference solves the
// systems of QOP_asqtad_invert_multi one restart at a time,
// lib/asqtad_invert_p.c:332-647).
//
// Each system runs its own reduced-precision reliable-update CG (int16
// links and site vectors, FP32 arithmetic, FP64 scalars and reductions,
// FP64 true-residual updates; the single-system method of mixed.cu), but the
// hop kernel reads every link once for all systems of a launch: the link
// stream (576-672 bytes per site) is shared, each system adds only its
// 16-byte input and output sites.  With 16 systems a hop moves ~1.1 KB per
// site instead of 16 x 0.6 KB, and the kernel becomes bound by FP32 issue
// rather than HBM.
//
// One iteration for all systems is four launches:
//   K1  t_j  = D_oe p_j                 (shared links; sums |t_j|^2)
//   K2  Ap_j = m_j^2 p_j - D_eo t_j     (shared links; sums |p_j|^2 -> alpha_j)
//   K3  x_j += alpha_j p_j, r_j -= alpha_j Ap_j   (|r_j|^2 -> beta_j, update test)
//   K4  p_j = r_j + beta_j p_j
// A system whose state flag is set (update requested, breakdown, converged)
// is skipped by every kernel; the host serves reliable updates between
// chunks of `chunk` iterations and retires converged systems.  The decode
// and arithmetic of a slot are those of the single-system int16 hop, so a
// system takes the same iterations alone or in a batch.
#include "solvers.cuh"
#include "reduce.cuh"
#include "dslash.cuh"
#include "prof.cuh"
#include "fields.cuh"
#include "mixed.cuh"
#include "bmma.cuh"
#include <algorithm>
#include <array>
#include <map>
#include <vector>
#include <cmath>

namespace qopb {

enum { MIX_DONE = 4 };

// link of one slot decoded to integer units; returns the factor that scales them
__device__ __forceinline__ float q16_link(const uint4 ua, const uint4 ub, const uint2 uc, float2 U[9]) {
  U[0] = make_float2(u16_lo(ua.x), u16_hi(ua.x)); U[1] = make_float2(u16_lo(ua.y), u16_hi(ua.y));
  U[2] = make_float2(u16_lo(ua.z), u16_hi(ua.z)); U[3] = make_float2(u16_lo(ua.w), u16_hi(ua.w));
  U[4] = make_float2(u16_lo(ub.x), u16_hi(ub.x)); U[5] = make_float2(u16_lo(ub.y), u16_hi(ub.y));
  U[6] = make_float2(u16_lo(ub.z), u16_hi(ub.z)); U[7] = make_float2(u16_lo(ub.w), u16_hi(ub.w));
  U[8] = make_float2(u16_lo(uc.x), u16_hi(uc.x));
  return __uint_as_float(uc.y) * (1.0f / 32767.0f);
}

// long link stored as two rows (units of |c|/32767) + det phase; row 2 is
// det * conj(row0 x row1), brought to the same units
__device__ __forceinline__ float q16_link_recon(const uint4 ua, const uint2 ub, const float phase, const float cl,
                                                float2 U[9]) {
  U[0] = make_float2(u16_lo(ua.x), u16_hi(ua.x)); U[1] = make_float2(u16_lo(ua.y), u16_hi(ua.y));
  U[2] = make_float2(u16_lo(ua.z), u16_hi(ua.z)); U[3] = make_float2(u16_lo(ua.w), u16_hi(ua.w));
  U[4] = make_float2(u16_lo(ub.x), u16_hi(ub.x)); U[5] = make_float2(u16_lo(ub.y), u16_hi(ub.y));
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

// the same two decodes with the (re, im) pairs formed by one packed add
__device__ __forceinline__ float q16_link_pk(const uint4 ua, const uint4 ub, const uint2 uc, float2 U[9]) {
  U[0] = u16_pair(ua.x); U[1] = u16_pair(ua.y); U[2] = u16_pair(ua.z); U[3] = u16_pair(ua.w);
  U[4] = u16_pair(ub.x); U[5] = u16_pair(ub.y); U[6] = u16_pair(ub.z); U[7] = u16_pair(ub.w);
  U[8] = u16_pair(uc.x);
  return __uint_as_float(uc.y) * (1.0f / 32767.0f);
}
__device__ __forceinline__ float q16_link_recon_pk(const uint4 ua, const uint2 ub, const float phase, const float cl,
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

// Blocks are (site block sb, system group grp) flattened with the group
// fastest, so the blocks that share a site block's links run together and
// the links come from HBM once.  Vectors are [system][Vh] int16 sites.
// BG systems per thread (and per block); MINB resident blocks per SM; UNR
// slots unrolled (NL: straight-line code; 1: a loop over the slots, less
// code and fewer registers); PK: the link pairs multiply pre-scaled,
// duplicated site components into two packed accumulators per row
// (q16_pk_mul in mixed.cuh) instead of the duplicated, negated link copies
template <int NL, int KIND, bool RECON, int BG, int MINB, int UNR = NL, bool PK = false>
__global__ void __launch_bounds__(QB, MINB)
k_bhop(uint4 *__restrict__ out, const uint4 *__restrict__ src, const unsigned char *__restrict__ lk,
       const uint4 *__restrict__ same, Geom g, NbrGeom ng, int p, MixState *st, int nsys, int ngrp, double *part,
       unsigned *count, float c_long) {
  const int grp = blockIdx.x % ngrp, sb = blockIdx.x / ngrp, nsb = gridDim.x / ngrp;
  const int tid = threadIdx.x;
  const i64 Vh = g.Vh;
  const int i = sb * QB + tid;
  const int j0 = grp * BG;
  bool act[BG];
  bool any = false;
#pragma unroll
  for (int b = 0; b < BG; b++) {
    act[b] = (j0 + b < nsys) && st[j0 + b].flag == 0;
    any = any || act[b];
  }
  if (!any) return;   // uniform over the group: no block of it reduces
  double acc[BG];
#pragma unroll
  for (int b = 0; b < BG; b++) acc[b] = 0.0;
  if (i < Vh) {
    int x[4];
    site_coords(g, i, p, x);
    const int x0 = x[0], x1 = x[1], x2 = x[2], x3 = x[3];
    const int lex = ((x0 * g.L[1] + x1) * g.L[2] + x2) * g.L[3] + x3;
    float2 a[BG][3], pt[PK ? BG : 1][3], ps[PK ? BG : 1][3];
#pragma unroll
    for (int b = 0; b < BG; b++) a[b][0] = a[b][1] = a[b][2] = make_float2(0.f, 0.f);
#pragma unroll
    for (int b = 0; b < (PK ? BG : 1); b++)
#pragma unroll
      for (int r = 0; r < 3; r++) pt[b][r] = ps[b][r] = make_float2(0.f, 0.f);
    const unsigned char *gl = lk + (size_t)sb * q16_block_bytes(NL, RECON);
#pragma unroll UNR
    for (int k = 0; k < NL; k++) {
      const unsigned char *ls = gl + q16_slot_off(k, RECON);
      float2 U[9];
      float sl;
      if (RECON && (k & 1)) {
        const uint4 ua = __ldcs(reinterpret_cast<const uint4 *>(ls) + tid);
        const uint2 ub = __ldcs(reinterpret_cast<const uint2 *>(ls + 16 * QB) + tid);
        const float ph = __ldcs(reinterpret_cast<const float *>(ls + 24 * QB) + tid);
        sl = PK ? q16_link_recon_pk(ua, ub, ph, c_long, U) : q16_link_recon(ua, ub, ph, c_long, U);
      } else {
        const uint4 ua = __ldcs(reinterpret_cast<const uint4 *>(ls) + tid);
        const uint4 ub = __ldcs(reinterpret_cast<const uint4 *>(ls + 16 * QB) + tid);
        const uint2 uc = __ldcs(reinterpret_cast<const uint2 *>(ls + 32 * QB) + tid);
        sl = PK ? q16_link_pk(ua, ub, uc, U) : q16_link(ua, ub, uc, U);
      }
      int nbi;
      if constexpr (UNR == NL) nbi = nbr_fast(ng, x, lex, slot_mu<NL>(k), slot_disp<NL>(k));
      else nbi = nbr_sel(ng, x0, x1, x2, x3, lex, slot_mu<NL>(k), slot_disp<NL>(k));
      uint4 nb[BG];
#pragma unroll
      for (int b = 0; b < BG; b++) nb[b] = act[b] ? src[(i64)(j0 + b) * Vh + nbi] : make_uint4(0, 0, 0, 0);
      if constexpr (PK) {
#pragma unroll
        for (int b = 0; b < BG; b++) {
          if (!act[b]) continue;
          float2 vx[3], vy[3];
          q16_pk_site(nb[b], sl, vx, vy);
          q16_pk_mul(U, vx, vy, pt[b], ps[b]);
        }
        continue;
      }
      // packed FP32x2 FMAs (sm_100): t += (Re u, Re u)(v.x, v.y) + (-Im u, Im u)(v.y, v.x)
      // rounds every lane exactly as the scalar complex FMA sequence does
      float2 ur[9], ui[9];
#pragma unroll
      for (int e = 0; e < 9; e++) {
        ur[e] = make_float2(U[e].x, U[e].x);
        ui[e] = make_float2(-U[e].y, U[e].y);
      }
#pragma unroll
      for (int b = 0; b < BG; b++) {
        if (!act[b]) continue;
        float2 v[3];
        const float sc = sl * SpQ16::raw(nb[b], v);
        const float2 sc2 = make_float2(sc, sc);
        const float2 w[3] = {make_float2(v[0].y, v[0].x), make_float2(v[1].y, v[1].x), make_float2(v[2].y, v[2].x)};
#pragma unroll
        for (int r = 0; r < 3; r++) {
          float2 t = make_float2(0.f, 0.f);
#pragma unroll
          for (int c = 0; c < 3; c++) {
            t = __ffma2_rn(ur[3 * r + c], v[c], t);
            t = __ffma2_rn(ui[3 * r + c], w[c], t);
          }
          a[b][r] = __ffma2_rn(sc2, t, a[b][r]);
        }
      }
    }
    if constexpr (PK) {
#pragma unroll
      for (int b = 0; b < BG; b++) q16_pk_rows(pt[b], ps[b], a[b]);
    }
#pragma unroll
    for (int b = 0; b < BG; b++) {
      if (!act[b]) continue;
      const i64 o = (i64)(j0 + b) * Vh;
      if (KIND == 1) {
        acc[b] = (double)a[b][0].x * a[b][0].x + (double)a[b][0].y * a[b][0].y + (double)a[b][1].x * a[b][1].x +
                 (double)a[b][1].y * a[b][1].y + (double)a[b][2].x * a[b][2].x + (double)a[b][2].y * a[b][2].y;
        SpQ16::store(out + o, i, Vh, a[b]);
      } else {
        const float m2 = (float)st[j0 + b].m2;
        float2 sv[3];
        SpQ16::load(same + o, i, Vh, sv);
#pragma unroll
        for (int c = 0; c < 3; c++) a[b][c] = make_float2(m2 * sv[c].x - a[b][c].x, m2 * sv[c].y - a[b][c].y);
        SpQ16::store(out + o, i, Vh, a[b]);
        acc[b] = (double)sv[0].x * sv[0].x + (double)sv[0].y * sv[0].y + (double)sv[1].x * sv[1].x +
                 (double)sv[1].y * sv[1].y + (double)sv[2].x * sv[2].x + (double)sv[2].y * sv[2].y;
      }
    }
  }
  __shared__ double res[BG];
  if (group_sum<BG>(acc, part + (size_t)grp * nsb * BG, count + grp, res, sb, nsb)) {
#pragma unroll
    for (int b = 0; b < BG; b++) {
      if (!act[b]) continue;
      MixState *s = st + j0 + b;
      if (KIND == 1) {
        s->dp2 = res[b];
      } else {
        const double pAp = s->dp2 + s->m2 * res[b];   // <p, A p> = |D p|^2 + m^2 |p|^2
        if (!(pAp > 0)) s->flag = MIX_BREAK;
        else s->alpha = s->rsq / pAp;
      }
    }
  }
}

// x_j += alpha_j p_j, r_j -= alpha_j Ap_j, |r_j|^2: blockIdx.y = system
__global__ void __launch_bounds__(256)
k_bupdate(float2 *__restrict__ xs, uint4 *__restrict__ r, const uint4 *__restrict__ p, const uint4 *__restrict__ Ap,
          i64 Vh, MixState *st, double *part, unsigned *count) {
  const int j = blockIdx.y;
  MixState *s = st + j;
  if (s->flag) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const i64 o = (i64)j * Vh;
  float2 *xj = xs + 3 * o;
  double acc1[1] = {0.0};
  if (i < Vh) {
    const float al = (float)s->alpha;
    float2 pv[3], av[3], rv[3];
    SpQ16::load(p + o, i, Vh, pv);
    SpQ16::load(Ap + o, i, Vh, av);
    SpQ16::load(r + o, i, Vh, rv);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float2 xv = xj[c * Vh + i];
      xv.x = fmaf(al, pv[c].x, xv.x);
      xv.y = fmaf(al, pv[c].y, xv.y);
      xj[c * Vh + i] = xv;
      rv[c].x = fmaf(-al, av[c].x, rv[c].x);
      rv[c].y = fmaf(-al, av[c].y, rv[c].y);
    }
    SpQ16::store(r + o, i, Vh, rv);
    acc1[0] = (double)rv[0].x * rv[0].x + (double)rv[0].y * rv[0].y + (double)rv[1].x * rv[1].x +
              (double)rv[1].y * rv[1].y + (double)rv[2].x * rv[2].x + (double)rv[2].y * rv[2].y;
  }
  if (grid_sum<1>(acc1, part + (size_t)j * gridDim.x, count + j, &s->red)) {
    const double rn = s->red;
    s->iter += 1;
    s->rsq_old = s->rsq;
    s->rsq = rn;
    s->beta = rn / s->rsq_old;
    if (rn > s->maxr2) s->maxr2 = rn;
    if (rn < s->delta2 * s->maxr2 || rn <= s->stop || s->iter >= s->max_iter) s->flag = MIX_UPDATE;
  }
}

// p_j = r_j + beta_j p_j: blockIdx.y = system
__global__ void __launch_bounds__(256)
k_bp(uint4 *__restrict__ p, const uint4 *__restrict__ r, i64 Vh, const MixState *st) {
  const int j = blockIdx.y;
  if (st[j].flag) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Vh) return;
  const i64 o = (i64)j * Vh;
  const float be = (float)st[j].beta;
  float2 pv[3], rv[3];
  SpQ16::load(p + o, i, Vh, pv);
  SpQ16::load(r + o, i, Vh, rv);
#pragma unroll
  for (int c = 0; c < 3; c++) pv[c] = make_float2(fmaf(be, pv[c].x, rv[c].x), fmaf(be, pv[c].y, rv[c].y));
  SpQ16::store(p + o, i, Vh, pv);
}

// batched hop variants (option batch_kernel): systems per thread, the
// register cap (resident blocks per SM) and the slot unrolling.  At 32^4
// with 16 systems a hop takes 531 us with variant 7 (8 systems per thread,
// 3 blocks per SM, slot loop unrolled by 2; the default), 557-580 us with
// 1, 6, 9, 10, 605-679 us with 0, 2, 3, 5, 622 us with 8 and 705-1074 us
// with 11 and 4 (16 / 8 systems, fully unrolled: ~240 registers).  The
// kernel issues ~60-90 instructions per system and slot at ~55% issue
// utilisation; HBM traffic equals the compulsory bytes (ncu), so it is
// instruction- and latency-bound, not HBM-bound.  12-15 use the packed pair
// form of the one-system hop (q16_pk_mul): 550 us with 4 systems per thread
// (12, against 577 for 1), but 625 / 810 us with 8 (13 / 14: two
// accumulators per row and system exceed the register budget), so 7 stays
// the choice for 16 systems; at 24^3x48 with 12 systems 12 and 1 tie
// (114.0 / 113.8 us).
struct BhopShape { int bg, minb; };
static const BhopShape kBhop[] = {{4, 1}, {4, 5}, {2, 8}, {2, 1}, {8, 1}, {4, 6}, {4, 5}, {8, 3}, {8, 2},
                                  {8, 3}, {8, 4}, {16, 2}, {4, 5}, {8, 3}, {8, 2}, {4, 4}};
constexpr int N_BHOP = (int)(sizeof(kBhop) / sizeof(kBhop[0]));

template <int KIND, int BG, int MINB, int UNR = 16, bool PK = false>
static void launch_bhop_t(int nl, bool recon, int ngrp, int nsb, uint4 *out, const uint4 *src,
                          const unsigned char *lk, const uint4 *same, const Geom &g, const NbrGeom &ng, int par,
                          MixState *st, int nsys, double *part, unsigned *count, float c_long) {
  Context &c = ctx();
  const int grid = ngrp * nsb;
#define BH_ARGS out, src, lk, same, g, ng, par, st, nsys, ngrp, part, count, c_long
  constexpr int U8 = UNR < 8 ? UNR : 8;
  if (nl != 16) k_bhop<8, KIND, false, BG, MINB, U8, PK><<<grid, QB, 0, c.s>>>(BH_ARGS);
  else if (recon) k_bhop<16, KIND, true, BG, MINB, UNR, PK><<<grid, QB, 0, c.s>>>(BH_ARGS);
  else k_bhop<16, KIND, false, BG, MINB, UNR, PK><<<grid, QB, 0, c.s>>>(BH_ARGS);
#undef BH_ARGS
}

template <int KIND>
static void launch_bhop(int variant, int nl, bool recon, int ngrp, int nsb, uint4 *out, const uint4 *src,
                        const unsigned char *lk, const uint4 *same, const Geom &g, const NbrGeom &ng, int par,
                        MixState *st, int nsys, double *part, unsigned *count, float c_long) {
#define BH_CALL(B, M, ...) launch_bhop_t<KIND, B, M, ##__VA_ARGS__>(nl, recon, ngrp, nsb, out, src, lk, same, g, ng, par, st, nsys, \
                                                part, count, c_long)
  switch (variant) {
    case 1: BH_CALL(4, 5); break;
    case 2: BH_CALL(2, 8); break;
    case 3: BH_CALL(2, 1); break;
    case 4: BH_CALL(8, 1); break;
    case 5: BH_CALL(4, 6); break;
    case 6: BH_CALL(4, 5, 2); break;   // slot loop unrolled by 2
    case 7: BH_CALL(8, 3, 2); break;
    case 8: BH_CALL(8, 2, 1); break;
    case 9: BH_CALL(8, 3, 4); break;
    case 10: BH_CALL(8, 4, 1); break;
    case 11: BH_CALL(16, 2, 1); break;
    case 12: BH_CALL(4, 5, 16, true); break;   // packed pairs (q16_pk_mul)
    case 13: BH_CALL(8, 3, 2, true); break;
    case 14: BH_CALL(8, 2, 1, true); break;
    case 15: BH_CALL(4, 4, 2, true); break;
    default: BH_CALL(4, 1); break;
  }
#undef BH_CALL
}

// autotuned batched hop variant per (lattice extents, links per site,
// long-link reconstruction, systems)
static std::map<std::array<int, 7>, int> g_bhop_tuned;

struct BatchEngine::Impl {
  FlaT<double> *f;
  int lat, eo, cap;
  i64 Vh;
  Range is;
  NbrGeom ng;
  int nsb, gridv;
  // vectors: int16 records [system][Vh], or with the tensor-core hop
  // (batch_kernel 16, tc) bf16 hi / lo records [Vh][16] (bmma.cuh)
  bool tc = false;
  uint4 *rs = nullptr, *ps = nullptr, *Aps = nullptr, *ts = nullptr;
  B16Rec *brs = nullptr, *bps = nullptr, *bAps = nullptr, *bts = nullptr;
  float2 *xs = nullptr;
  c2<double> *r = nullptr, *Ax = nullptr, *tmp = nullptr;
  double *part = nullptr;
  unsigned *count = nullptr;
  MixState *dst = nullptr;
  MixState *h = nullptr;     // host copy of the per-slot solver state (pinned: source of the uploads)
  MixState *hd = nullptr;    // pinned landing buffer of the download after a chunk
  cudaStream_t own = nullptr;
  bool inflight = false;     // a chunk was launched and not yet collected
  int launched_n = 0;
  std::vector<int> recs;
  struct Sys {
    bool busy = false;
    c2<double> *x = nullptr;
    const c2<double> *b = nullptr;
    double mass = 0, b2 = 0, r2 = 0;
    int nru = 0, stalls = 0, last_iter = 0;
  };
  std::vector<Sys> sys;
  std::vector<int> done_now;   // started at their target: reported by the next step
  static size_t npart(int cap, int nsb, int gridv, bool tc) {
    // k_bhop: (groups x BG <= cap + 15) x site blocks; k_bupdate: cap x gridv;
    // the tensor-core kernels: 16 per block
    if (tc) return bmma_part_doubles();
    return std::max<size_t>((size_t)(cap + 15) * nsb, (size_t)cap * gridv);
  }
  void release_all() {
    if (own) cudaStreamSynchronize(own);   // nothing of ours in flight when the memory goes back
    dfree(rs); dfree(ps); dfree(Aps); dfree(ts); dfree(xs); dfree(r); dfree(Ax); dfree(tmp);
    dfree(brs); dfree(bps); dfree(bAps); dfree(bts);
    dfree(part); dfree(count); dfree(dst);
    if (h) cudaFreeHost(h);
    if (hd) cudaFreeHost(hd);
    if (own) cudaStreamDestroy(own);
    h = hd = nullptr;
    own = nullptr;
  }
  void check_current() const {
    if (ctx().lat != lat) fail(QOP_FAIL, "batched solver: its lattice %d is not the current one", lat);
  }
  // FP64 true residual b_j - A_j x_j into r; returns its norm^2
  double true_resid(int j) {
    LinOp<double> L{f, sys[j].mass, eo, tmp};
    L.d2(Ax, sys[j].x);
    Blas<double>::axpby(r, 1.0, sys[j].b, -1.0, Ax, is);
    return Blas<double>::norm2(r, is);
  }
};

static bool use_tc() { return ctx().opt.batch_kernel == 16; }

size_t BatchEngine::bytes(const Geom &g, int cap) {
  const int nsb = (int)((g.Vh + QB - 1) / QB), gridv = grid_for(g.Vh, 256);
  const bool tc = use_tc();
  const size_t vec = tc ? (size_t)BSYS * g.Vh * (4 * sizeof(B16Rec) + 3 * sizeof(float2))
                        : (size_t)cap * g.Vh * (4 * sizeof(uint4) + 3 * sizeof(float2));
  return vec + 3 * sizeof(c2<double>) * vec_elems(g) + sizeof(double) * Impl::npart(cap, nsb, gridv, tc) +
         (sizeof(unsigned) + sizeof(MixState)) * cap;
}

BatchEngine::BatchEngine(FlaT<double> *f, int eo, int cap, bool own_stream) : d(new Impl()) {
  Impl &e = *d;
  Context &c = ctx();
  const Geom &g = c.g;
  if (cap < 1 || cap > BATCH_MAX) {
    delete d;
    fail(QOP_FAIL, "batched solver: %d slots (1..%d)", cap, BATCH_MAX);
  }
  e.f = f;
  e.lat = c.lat;
  e.eo = eo;
  e.cap = cap;
  e.Vh = g.Vh;
  e.is = vrange(g, eo);
  for (int k = 0; k < 4; k++) e.ng.L[k] = g.L[k];
  e.ng.str[3] = 1; e.ng.str[2] = g.L[3]; e.ng.str[1] = g.L[2] * g.L[3]; e.ng.str[0] = g.L[1] * g.L[2] * g.L[3];
  e.nsb = (int)((e.Vh + QB - 1) / QB);
  e.gridv = grid_for(e.Vh, 256);
  e.sys.assign(cap, Impl::Sys{});
  try {
    QCHECK(cudaMallocHost(&e.h, sizeof(MixState) * cap));
    QCHECK(cudaMallocHost(&e.hd, sizeof(MixState) * cap));
    for (int j = 0; j < cap; j++) {
      e.h[j] = MixState{};
      e.h[j].flag = MIX_DONE;   // free slots are skipped by every kernel
    }
    sloppy_get(f, LK_Q16);   // the int16 link copy, built on first use
    const i64 Vh = e.Vh;
    e.tc = use_tc();
    if (e.tc) {
      e.brs = dalloc<B16Rec>(BSYS * Vh);
      e.bps = dalloc<B16Rec>(BSYS * Vh);
      e.bAps = dalloc<B16Rec>(BSYS * Vh);
      e.bts = dalloc<B16Rec>(BSYS * Vh);
      e.xs = dalloc<float2>(3 * BSYS * Vh);
      dzero(e.xs, sizeof(float2) * 3 * BSYS * Vh);
    } else {
      e.rs = dalloc<uint4>(cap * Vh);
      e.ps = dalloc<uint4>(cap * Vh);
      e.Aps = dalloc<uint4>(cap * Vh);
      e.ts = dalloc<uint4>(cap * Vh);
      e.xs = dalloc<float2>(3 * cap * Vh);
      dzero(e.xs, sizeof(float2) * 3 * cap * Vh);
    }
    e.r = dalloc<c2<double>>(vec_elems(g));
    e.Ax = dalloc<c2<double>>(vec_elems(g));
    e.tmp = dalloc<c2<double>>(vec_elems(g));
    e.part = dalloc<double>(Impl::npart(cap, e.nsb, e.gridv, e.tc));
    e.count = dalloc<unsigned>(cap);
    dzero(e.count, sizeof(unsigned) * cap);
    e.dst = dalloc<MixState>(cap);
    // the allocations and the link copy are complete before any other
    // stream uses them
    sync();
    if (own_stream) QCHECK(cudaStreamCreateWithFlags(&e.own, cudaStreamNonBlocking));
  } catch (...) {
    e.release_all();
    delete d;
    throw;
  }
}

BatchEngine::~BatchEngine() {
  d->release_all();
  delete d;
}

int BatchEngine::cap() const { return d->cap; }
cudaStream_t BatchEngine::stream() const { return d->own ? d->own : ctx().s; }
int BatchEngine::busy() const {
  int n = 0;
  for (const auto &y : d->sys) n += y.busy;
  return n;
}
int BatchEngine::running() const {
  int n = 0;
  for (int j = 0; j < d->cap; j++) n += d->sys[j].busy && d->h[j].flag != MIX_DONE;
  return n;
}
bool BatchEngine::running(int s) const {
  return s >= 0 && s < d->cap && d->sys[s].busy && d->h[s].flag != MIX_DONE;
}
int BatchEngine::free_slot() const {
  for (int j = 0; j < d->cap; j++)
    if (!d->sys[j].busy) return j;
  return -1;
}
int BatchEngine::iters(int s) const { return d->h[s].iter + d->sys[s].nru; }
double BatchEngine::final_rsq(int s) const { return d->sys[s].b2 > 0 ? d->sys[s].r2 / d->sys[s].b2 : 0.0; }

void BatchEngine::fold(int s) {
  Impl &e = *d;
  StreamScope ss(e.own);
  if (s < 0 || s >= e.cap || !e.sys[s].busy) return;
  if (e.inflight) fail(QOP_FAIL, "batched solver: a chunk is in flight");
  const Context &c = ctx();
  const i64 Vh = e.Vh;
  if (e.tc) k_b16_fold_x<<<e.gridv, 256, 0, c.s>>>(e.sys[s].x + e.is.off, e.xs, s, Vh);
  else k_fold_x<<<grid_for(3 * Vh, 256), 256, 0, c.s>>>(e.sys[s].x + e.is.off, e.xs + 3 * s * Vh, 3 * Vh);
  QLAUNCH();
}

void BatchEngine::release(int s) {
  if (s < 0 || s >= d->cap) return;
  d->sys[s] = Impl::Sys{};
  d->h[s] = MixState{};
  d->h[s].flag = MIX_DONE;
}

void BatchEngine::start(int s, c2<double> *x, const c2<double> *b, double mass, double rsqmin, int max_iter,
                        bool x_zero) {
  Impl &e = *d;
  StreamScope ss(e.own);
  Context &c = ctx();
  e.check_current();
  if (s < 0 || s >= e.cap || e.sys[s].busy) fail(QOP_FAIL, "batched solver: slot %d is not free", s);
  if (e.inflight) fail(QOP_FAIL, "batched solver: a chunk is in flight");
  sync();   // the last upload of the slot states has read them
  const i64 Vh = e.Vh;
  need_finite(Blas<double>::norm2(b, e.is), "batched solver: source norm");   // before the slot is taken
  Impl::Sys &y = e.sys[s];
  y = Impl::Sys{};
  y.busy = true;
  y.x = x;
  y.b = b;
  y.mass = mass;
  MixState &st = e.h[s];
  st = MixState{};
  y.b2 = Blas<double>::norm2(b, e.is);
  st.stop = rsqmin * y.b2;
  st.delta2 = c.opt.ru_delta * c.opt.ru_delta;
  st.m2 = mass * mass;
  st.max_iter = max_iter;
  if (y.b2 == 0.0 || x_zero) Blas<double>::zero(x, e.is);
  y.r2 = y.b2 == 0.0 ? 0.0 : x_zero ? y.b2 : e.true_resid(s);
  if (y.b2 == 0.0 || y.r2 <= st.stop) {
    st.flag = MIX_DONE;
    e.done_now.push_back(s);
    return;
  }
  if (e.tc) {
    k_b16_from_f64<<<e.gridv, 256, 0, c.s>>>(e.brs, s, (x_zero ? b : e.r) + e.is.off, Vh);
    k_b16_copy_sys<<<e.gridv, 256, 0, c.s>>>(e.bps, e.brs, s, Vh);
    k_b16_zero_x<<<e.gridv, 256, 0, c.s>>>(e.xs, s, Vh);
    QLAUNCHN(3);
  } else {
    k_to_sloppy<SpQ16><<<e.gridv, 256, 0, c.s>>>(e.rs + s * Vh, (x_zero ? b : e.r) + e.is.off, Vh);
    k_copy_elems<uint4><<<grid_for(Vh, 256), 256, 0, c.s>>>(e.ps + s * Vh, e.rs + s * Vh, Vh);
    QLAUNCHN(2);
    dzero(e.xs + 3 * s * Vh, sizeof(float2) * 3 * Vh);
  }
  st.rsq = st.rsq_old = st.maxr2 = y.r2;
  st.flag = MIX_RUN;
}

std::vector<int> BatchEngine::step() {
  launch();
  return collect();
}

void BatchEngine::launch() {
  Impl &e = *d;
  StreamScope ss(e.own);
  Context &c = ctx();
  e.check_current();
  if (e.inflight) fail(QOP_FAIL, "batched solver: a chunk is in flight");
  const Geom &g = c.g;
  const i64 Vh = e.Vh;
  const int eo = e.eo, p = eo, q = 1 - eo;
  int n = 0, active = 0;   // launches cover slots 0 .. n-1
  for (int j = 0; j < e.cap; j++)
    if (e.sys[j].busy) {
      n = j + 1;
      active += e.h[j].flag != MIX_DONE;
    }
  if (active == 0) return;
  SloppyLinks *sl = sloppy_get(e.f, LK_Q16);
  const LinksSloppy lk_p = links_parity(sl, LK_Q16, p), lk_q = links_parity(sl, LK_Q16, q);
  const int nl = sl->nl;
  const bool recon = sl->recon != 0;
  const float c_long = (float)sl->c_long;
  const int nsb = e.nsb, gridv = e.gridv;
  QCHECK(cudaMemcpyAsync(e.dst, e.h, sizeof(MixState) * n, cudaMemcpyHostToDevice, c.s));
  // by default 8 systems per thread when they fill whole groups of 8 (16
  // sources at 32^4: 531 us per hop against 574 with 4), else 4 (12 masses
  // at 24^3x48: 1696 ms per call against 1989 ms with groups of 8 and 4);
  // batch_kernel -2: the fastest of 1, 6, 7, 9, 12 timed on the first step
  // with this lattice and number of systems
  const double link_site = recon ? (nl / 2) * (40.0 + 28.0) : nl * 40.0;
  const int chunk = c.opt.chunk;
  std::vector<int> recs;
  if (e.tc) {
    // tensor-core hop: bf16 hi / lo records of 24 bytes per system and site
    char tname[32];
    snprintf(tname, sizeof tname, "bhop_mma_x%d", n);
    const double tb = (double)Vh * (link_site + 2.0 * 24 * active);
    for (int k = 0; k < chunk; k++) {
      {
        ProfScope s1(tname, tb);
        launch_bmma_hop(1, nl, recon, c_long, e.bts, e.bps, (const unsigned char *)lk_q.a, nullptr, g, e.ng, q, e.dst,
                        n, e.part, e.count);
        QLAUNCH();
        recs.push_back(s1.idx);
      }
      {
        ProfScope s2(tname, tb + (double)Vh * 24 * active);
        launch_bmma_hop(2, nl, recon, c_long, e.bAps, e.bts, (const unsigned char *)lk_p.a, e.bps, g, e.ng, p,
                        e.dst, n, e.part, e.count);
        QLAUNCH();
        recs.push_back(s2.idx);
      }
      launch_b16_update(e.xs, e.brs, e.bps, e.bAps, Vh, e.dst, n, e.part, e.count);
      launch_b16_p(e.bps, e.brs, Vh, e.dst, n);
      QLAUNCHN(2);
    }
    QCHECK(cudaMemcpyAsync(e.hd, e.dst, sizeof(MixState) * n, cudaMemcpyDeviceToHost, c.s));
    e.recs.swap(recs);
    e.launched_n = n;
    e.inflight = true;
    return;
  }
  int variant = c.opt.batch_kernel == -1 ? (n % 8 == 0 ? 7 : 1) : std::min(c.opt.batch_kernel, N_BHOP - 1);
  if (c.opt.batch_kernel == -2) {
    const std::array<int, 7> key{g.L[0], g.L[1], g.L[2], g.L[3], nl, recon ? 1 : 0, n};
    auto it = g_bhop_tuned.find(key);
    if (it != g_bhop_tuned.end()) {
      variant = it->second;
    } else {
      const unsigned char *lq = (const unsigned char *)lk_q.a;
      variant = tune_pick({1, 6, 7, 9, 12}, [&](int v) {   // t = D p: recomputed by the first iteration
        launch_bhop<1>(v, nl, recon, (n + kBhop[v].bg - 1) / kBhop[v].bg, nsb, e.ts, e.ps, lq, nullptr, g, e.ng, q,
                       e.dst, n, e.part, e.count, c_long);
        QLAUNCH();
      });
      g_bhop_tuned[key] = variant;
      log0(QOP_VERB_LOW, "autotune: batched hop variant %d for %d systems on %dx%dx%dx%d\n", variant, n, g.L[0],
           g.L[1], g.L[2], g.L[3]);
    }
  }
  const int BG = kBhop[variant].bg;
  const int ngrp = (n + BG - 1) / BG;
  char hname[32];
  snprintf(hname, sizeof hname, "bhop_q16_x%d", active);   // timing class: systems running in the launch
  // compulsory bytes of one hop for the systems running in this chunk
  const double hop_bytes = (double)Vh * (link_site + 2.0 * 16 * active);
  for (int k = 0; k < chunk; k++) {
    {
      ProfScope s1(hname, hop_bytes);
      launch_bhop<1>(variant, nl, recon, ngrp, nsb, e.ts, e.ps, (const unsigned char *)lk_q.a, nullptr, g, e.ng, q,
                     e.dst, n, e.part, e.count, c_long);
      recs.push_back(s1.idx);
    }
    {
      ProfScope s2(hname, hop_bytes + (double)Vh * 16 * active);
      launch_bhop<2>(variant, nl, recon, ngrp, nsb, e.Aps, e.ts, (const unsigned char *)lk_p.a, e.ps, g, e.ng, p,
                     e.dst, n, e.part, e.count, c_long);
      recs.push_back(s2.idx);
    }
    k_bupdate<<<dim3(gridv, n), 256, 0, c.s>>>(e.xs, e.rs, e.ps, e.Aps, Vh, e.dst, e.part, e.count);
    k_bp<<<dim3(gridv, n), 256, 0, c.s>>>(e.ps, e.rs, Vh, e.dst);
    QLAUNCHN(4);
  }
  QCHECK(cudaMemcpyAsync(e.hd, e.dst, sizeof(MixState) * n, cudaMemcpyDeviceToHost, c.s));
  e.recs.swap(recs);
  e.launched_n = n;
  e.inflight = true;
}

std::vector<int> BatchEngine::collect() {
  Impl &e = *d;
  StreamScope ss(e.own);
  Context &c = ctx();
  e.check_current();
  std::vector<int> fin;
  fin.swap(e.done_now);
  if (!e.inflight) return fin;
  e.inflight = false;
  const i64 Vh = e.Vh;
  const int n = e.launched_n, gridv = e.gridv;
  std::vector<int> recs;
  recs.swap(e.recs);
  sync();
  memcpy(e.h, e.hd, sizeof(MixState) * n);   // the states after the chunk
  MixState *h = e.h;
  // drop timing records of hops that found every system idle
  int most = 0;
  for (int j = 0; j < n; j++)
    if (e.sys[j].busy) most = std::max(most, h[j].iter - e.sys[j].last_iter + (h[j].flag == MIX_BREAK ? 1 : 0));
  for (size_t k = 2 * (size_t)most; k < recs.size(); k++) prof_discard(recs[k]);
  std::vector<int> pupd;
  for (int j = 0; j < n; j++) {
    Impl::Sys &y = e.sys[j];
    MixState &s = h[j];
    if (!y.busy) continue;
    const int ran = s.iter - y.last_iter;
    y.last_iter = s.iter;
    if (s.flag != MIX_UPDATE && s.flag != MIX_BREAK) continue;
    y.stalls = ran == 0 ? y.stalls + 1 : 0;   // repeated breakdown without progress
    // reliable update: fold the sloppy solution into FP64, true residual
    if (e.tc) k_b16_fold_x<<<gridv, 256, 0, c.s>>>(y.x + e.is.off, e.xs, j, Vh);
    else k_fold_x<<<grid_for(3 * Vh, 256), 256, 0, c.s>>>(y.x + e.is.off, e.xs + 3 * j * Vh, 3 * Vh);
    QLAUNCH();
    y.r2 = e.true_resid(j);
    need_finite(y.r2, "batched solver: true residual norm");
    y.nru++;
    log0(QOP_VERB_MED, "BATCHCG[%d/%d]: iter %d sloppy rsq %g true rsq %g (stop %g)\n", j, n, s.iter, s.rsq, y.r2,
         s.stop);
    if (y.r2 <= s.stop || s.iter + y.nru >= s.max_iter || y.stalls > 2) {
      s.flag = MIX_DONE;
      fin.push_back(j);
      continue;
    }
    const bool broke = s.flag == MIX_BREAK || !(s.rsq_old > 0);
    const double rsq_prev = s.rsq_old;
    if (e.tc) k_b16_from_f64<<<gridv, 256, 0, c.s>>>(e.brs, j, e.r + e.is.off, Vh);
    else k_to_sloppy<SpQ16><<<gridv, 256, 0, c.s>>>(e.rs + j * Vh, e.r + e.is.off, Vh);
    QLAUNCH();
    s.rsq = y.r2;
    s.maxr2 = y.r2;
    s.flag = MIX_RUN;
    if (broke) {   // restart the recursion from the true residual
      if (e.tc) k_b16_copy_sys<<<gridv, 256, 0, c.s>>>(e.bps, e.brs, j, Vh);
      else k_copy_elems<uint4><<<grid_for(Vh, 256), 256, 0, c.s>>>(e.ps + j * Vh, e.rs + j * Vh, Vh);
      QLAUNCH();
    } else {
      s.beta = y.r2 / rsq_prev;
      pupd.push_back(j);
    }
  }
  QCHECK(cudaMemcpyAsync(e.dst, h, sizeof(MixState) * n, cudaMemcpyHostToDevice, c.s));
  for (int j : pupd) {
    if (e.tc) launch_b16_p(e.bps, e.brs, Vh, e.dst, n, j);
    else k_bp<<<dim3(gridv, 1), 256, 0, c.s>>>(e.ps + j * Vh, e.rs + j * Vh, Vh, e.dst + j);
    QLAUNCH();
  }
  return fin;
}

void run_batch(FlaT<double> *f, int eo, int n, const double *mass, c2<double> **x, c2<double> *const *b,
               const double *rsqmin, int max_iter, int *iters, double *final_rsq) {
  if (n < 1) return;
  if (n > BATCH_MAX) fail(QOP_FAIL, "run_batch: %d systems exceed the batch limit %d", n, BATCH_MAX);
  // With option batch_tail, the last system still running leaves the batch
  // and finishes in the one-system solver (its fused kernels cost about a
  // third of a batched hop that carries one system): the correction
  // A e = b - A x from its current x, to the same FP64 target.
  const bool tail_ok = ctx().opt.batch_tail && n > 1 && !use_tc();
  int tail = -1;
  {
    BatchEngine e(f, eo, n);
    for (int j = 0; j < n; j++) e.start(j, x[j], b[j], mass[j], rsqmin[j], max_iter, false);
    for (int left = n; left > 0;) {
      const int k = (int)e.step().size();
      if (k == 0 && e.running() == 0) break;
      left -= k;
      if (tail_ok && left == 1 && e.running() == 1) {
        for (int j = 0; j < n; j++)
          if (e.running(j)) tail = j;
        break;
      }
    }
    if (tail >= 0) e.fold(tail);
    for (int j = 0; j < n; j++) {
      iters[j] = e.iters(j);
      final_rsq[j] = e.final_rsq(j);
    }
    sync();
  }
  if (tail < 0) return;
  const Geom &g = ctx().g;
  const Range is = vrange(g, eo);
  ScopedVecs own;
  c2<double> *r = own.add(), *ex = own.add(), *tmp = own.add();
  LinOp<double> L{f, mass[tail], eo, tmp};
  L.d2(r, x[tail]);
  Blas<double>::axpby(r, 1.0, b[tail], -1.0, r, is);   // r = b - A x
  const double b2 = Blas<double>::norm2(b[tail], is), r2 = Blas<double>::norm2(r, is);
  need_finite(r2, "batched solver: residual of the last system");
  if (!(r2 > rsqmin[tail] * b2)) {   // converged at the hand-off
    final_rsq[tail] = b2 > 0 ? r2 / b2 : 0.0;
    return;
  }
  QOP_invert_arg_t ia = QOP_INVERT_ARG_DEFAULT;
  ia.max_iter = std::max(1, max_iter - iters[tail]);
  ia.evenodd = (QOP_evenodd_t)eo;
  QOP_resid_arg_t ra = QOP_RESID_ARG_DEFAULT;
  ra.rsqmin = rsqmin[tail] * b2 / r2;
  QOP_resid_arg_t *rap = &ra;
  const double zero = 0.0;
  mixed_cgms(L, &ia, &rap, &zero, 1, &ex, r, eo, 16);
  Blas<double>::axpy(x[tail], 1.0, ex, is);   // x += e
  iters[tail] += ra.final_iter;
  final_rsq[tail] = ra.final_rsq * r2 / b2;
  sync();
}

}  // namespace qopb

namespace qopb {
__global__ void k_q16_to_f64(double2 *d, const uint4 *s, i64 Vh);   // mixed.cu
}

// the check below for the tensor-core format (batch_kernel 16): p_j split
// into bf16 hi / lo records, the two MMA hops, t_j and Ap_j decoded
static int sloppy_ddagd_batch_tc(QOP_info_t *info, qopb::FlaT<double> *f, int n, const double *masses,
                                 QOP_D3_ColorVector **t_out, QOP_D3_ColorVector **ap_out, QOP_D3_ColorVector **in,
                                 QOP_evenodd_t eo, double *sums) {
  using namespace qopb;
  B16Rec *ps = nullptr, *ts = nullptr, *as = nullptr;
  MixState *dst = nullptr;
  double *part = nullptr;
  unsigned *count = nullptr;
  auto release = [&]() { dfree(ps); dfree(ts); dfree(as); dfree(dst); dfree(part); dfree(count); };
  try {
    Context &c = ctx();
    const Geom &g = c.g;
    const i64 Vh = g.Vh;
    const int p = eo, q = 1 - eo, gridv = grid_for(Vh, 256);
    SloppyLinks *sl = sloppy_get(f, LK_Q16);
    const LinksSloppy lk_p = links_parity(sl, LK_Q16, p), lk_q = links_parity(sl, LK_Q16, q);
    ps = dalloc<B16Rec>(BSYS * Vh);
    ts = dalloc<B16Rec>(BSYS * Vh);
    as = dalloc<B16Rec>(BSYS * Vh);
    dst = dalloc<MixState>(n);
    part = dalloc<double>(bmma_part_doubles());
    count = dalloc<unsigned>(1);
    dzero(count, sizeof(unsigned));
    std::vector<MixState> h(n);
    for (int j = 0; j < n; j++) {
      h[j] = MixState{};
      h[j].flag = MIX_RUN;
      h[j].m2 = masses[j] * masses[j];
      h[j].rsq = h[j].rsq_old = h[j].maxr2 = 1.0;
      h[j].max_iter = 1 << 30;
      k_b16_from_f64<<<gridv, 256, 0, c.s>>>(ps, j, reinterpret_cast<VecT<double> *>(in[j])->d + par_off(g, p), Vh);
      QLAUNCH();
    }
    QCHECK(cudaMemcpyAsync(dst, h.data(), sizeof(MixState) * n, cudaMemcpyHostToDevice, c.s));
    NbrGeom ng;
    for (int d = 0; d < 4; d++) ng.L[d] = g.L[d];
    ng.str[3] = 1; ng.str[2] = g.L[3]; ng.str[1] = g.L[2] * g.L[3]; ng.str[0] = g.L[1] * g.L[2] * g.L[3];
    const double tb = (double)Vh * ((sl->recon ? (sl->nl / 2) * (40.0 + 28.0) : sl->nl * 40.0) + 2.0 * 24 * n);
    {
      ProfScope s1("check_bhop_mma", tb);
      launch_bmma_hop(1, sl->nl, sl->recon != 0, (float)sl->c_long, ts, ps, (const unsigned char *)lk_q.a, nullptr,
                      g, ng, q, dst, n, part, count);
      QLAUNCH();
    }
    {
      ProfScope s2("check_bhop_mma", tb + (double)Vh * 24 * n);
      launch_bmma_hop(2, sl->nl, sl->recon != 0, (float)sl->c_long, as, ts, (const unsigned char *)lk_p.a, ps, g,
                      ng, p, dst, n, part, count);
      QLAUNCH();
    }
    for (int j = 0; j < n; j++) {
      k_b16_to_f64<<<gridv, 256, 0, c.s>>>(reinterpret_cast<VecT<double> *>(t_out[j])->d + par_off(g, q), ts, j, Vh);
      k_b16_to_f64<<<gridv, 256, 0, c.s>>>(reinterpret_cast<VecT<double> *>(ap_out[j])->d + par_off(g, p), as, j, Vh);
      QLAUNCHN(2);
    }
    QCHECK(cudaMemcpyAsync(h.data(), dst, sizeof(MixState) * n, cudaMemcpyDeviceToHost, c.s));
    sync();
    if (sums)
      for (int j = 0; j < n; j++) {
        sums[2 * j] = h[j].dp2;
        sums[2 * j + 1] = h[j].alpha > 0 ? 1.0 / h[j].alpha : 0.0;
      }
    release();
    if (info) info->status = QOP_SUCCESS;
    return 0;
  } catch (Fail &e) {
    release();
    fprintf(stderr, "QOPB_D3_sloppy_ddagd_batch: %s\n", e.msg.c_str());
    if (info) info->status = e.status;
    return -1;
  }
}

// The batched reduced-precision operator of the batched solver, applied
// once with its own hop kernels to n <= 16 systems: p_j = sloppy(in_j) on
// parity eo, t_j = D_oe p_j, Ap_j = m_j^2 p_j - D_eo t_j; t_j and Ap_j are
// decoded into t_out[j] / ap_out[j].  sums[2j], sums[2j+1] = |t_j|^2 and
// <p_j, A_j p_j> = |t_j|^2 + m_j^2 |p_j|^2 as the kernels reduced them.
// variant: a batch_kernel value (0..15: int16 vectors; 16: the tensor-core
// hop on bf16 hi / lo vectors), or -1 for the solver's default choice for n
// systems.  Restates QOP_asqtad_ddagd_norm2 (lib/asqtad_dslash_p.c:1121-1138)
// for several vectors at once, as the reference's vectorised hop does
// (lib/asqtad_dslash_p.c:1246-1279); it exists so that the batched sloppy
// operator can be compared site by site with FP64.
extern "C" int QOPB_D3_sloppy_ddagd_batch(QOP_info_t *info, QOP_D3_FermionLinksAsqtad *asqtad, int n,
                                          const double *masses, QOP_D3_ColorVector **t_out,
                                          QOP_D3_ColorVector **ap_out, QOP_D3_ColorVector **in, QOP_evenodd_t eo,
                                          int variant, double *sums) {
  using namespace qopb;
  uint4 *ps = nullptr, *ts = nullptr, *as = nullptr;
  MixState *dst = nullptr;
  double *part = nullptr;
  unsigned *count = nullptr;
  auto release = [&]() { dfree(ps); dfree(ts); dfree(as); dfree(dst); dfree(part); dfree(count); };
  try {
    require_init("QOPB_D3_sloppy_ddagd_batch");
    dd_refuse("QOPB_D3_sloppy_ddagd_batch");
    handle_check(asqtad, "FermionLinksAsqtad");
    if (n < 1 || n > BATCH_MAX) fail(QOP_FAIL, "QOPB_D3_sloppy_ddagd_batch: %d systems (1..%d)", n, BATCH_MAX);
    if (!masses || !t_out || !ap_out || !in) fail(QOP_FAIL, "QOPB_D3_sloppy_ddagd_batch: NULL array");
    for (int j = 0; j < n; j++) {
      handle_check(t_out[j], "ColorVector");
      handle_check(ap_out[j], "ColorVector");
      handle_check(in[j], "ColorVector");
    }
    if (eo != QOP_EVEN && eo != QOP_ODD) fail(QOP_FAIL, "QOPB_D3_sloppy_ddagd_batch: eo must be EVEN or ODD");
    if (variant < -1 || variant > N_BHOP)
      fail(QOP_FAIL, "QOPB_D3_sloppy_ddagd_batch: variant %d (-1..%d)", variant, N_BHOP);
    if (variant == N_BHOP)
      return sloppy_ddagd_batch_tc(info, reinterpret_cast<FlaT<double> *>(asqtad), n, masses, t_out, ap_out, in, eo,
                                   sums);
    if (variant < 0) variant = n % 8 == 0 ? 7 : 1;
    FlaT<double> *f = reinterpret_cast<FlaT<double> *>(asqtad);
    Context &c = ctx();
    const Geom &g = c.g;
    const i64 Vh = g.Vh;
    const int p = eo, q = 1 - eo;
    SloppyLinks *sl = sloppy_get(f, LK_Q16);
    const LinksSloppy lk_p = links_parity(sl, LK_Q16, p), lk_q = links_parity(sl, LK_Q16, q);
    const int nsb = (int)((Vh + QB - 1) / QB), gridv = grid_for(Vh, 256);
    const int BG = kBhop[variant].bg, ngrp = (n + BG - 1) / BG;
    ps = dalloc<uint4>(n * Vh);
    ts = dalloc<uint4>(n * Vh);
    as = dalloc<uint4>(n * Vh);
    dst = dalloc<MixState>(n);
    part = dalloc<double>((size_t)ngrp * BG * nsb);
    count = dalloc<unsigned>(ngrp);
    dzero(count, sizeof(unsigned) * ngrp);
    std::vector<MixState> h(n);
    for (int j = 0; j < n; j++) {
      h[j] = MixState{};
      h[j].flag = MIX_RUN;
      h[j].m2 = masses[j] * masses[j];
      h[j].rsq = h[j].rsq_old = h[j].maxr2 = 1.0;
      h[j].max_iter = 1 << 30;
      k_to_sloppy<SpQ16><<<gridv, 256, 0, c.s>>>(ps + j * Vh, reinterpret_cast<VecT<double> *>(in[j])->d + par_off(g, p),
                                                 Vh);
      QLAUNCH();
    }
    QCHECK(cudaMemcpyAsync(dst, h.data(), sizeof(MixState) * n, cudaMemcpyHostToDevice, c.s));
    NbrGeom ng;
    for (int d = 0; d < 4; d++) ng.L[d] = g.L[d];
    ng.str[3] = 1; ng.str[2] = g.L[3]; ng.str[1] = g.L[2] * g.L[3]; ng.str[0] = g.L[1] * g.L[2] * g.L[3];
    const bool recon = sl->recon != 0;
    const float c_long = (float)sl->c_long;
    const double tb = (double)Vh * ((recon ? (sl->nl / 2) * (40.0 + 28.0) : sl->nl * 40.0) + 2.0 * 16 * n);
    {
      ProfScope s1("check_bhop_q16", tb);
      launch_bhop<1>(variant, sl->nl, recon, ngrp, nsb, ts, ps, (const unsigned char *)lk_q.a, nullptr, g, ng, q, dst,
                     n, part, count, c_long);
      QLAUNCH();
    }
    {
      ProfScope s2("check_bhop_q16", tb + (double)Vh * 16 * n);
      launch_bhop<2>(variant, sl->nl, recon, ngrp, nsb, as, ts, (const unsigned char *)lk_p.a, ps, g, ng, p, dst, n,
                     part, count, c_long);
      QLAUNCH();
    }
    for (int j = 0; j < n; j++) {
      k_q16_to_f64<<<gridv, 256, 0, c.s>>>(reinterpret_cast<VecT<double> *>(t_out[j])->d + par_off(g, q), ts + j * Vh,
                                          Vh);
      k_q16_to_f64<<<gridv, 256, 0, c.s>>>(reinterpret_cast<VecT<double> *>(ap_out[j])->d + par_off(g, p),
                                          as + j * Vh, Vh);
      QLAUNCHN(2);
    }
    QCHECK(cudaMemcpyAsync(h.data(), dst, sizeof(MixState) * n, cudaMemcpyDeviceToHost, c.s));
    sync();
    if (sums)
      for (int j = 0; j < n; j++) {
        sums[2 * j] = h[j].dp2;
        sums[2 * j + 1] = h[j].alpha > 0 ? 1.0 / h[j].alpha : 0.0;   // alpha = rsq / pAp with rsq = 1
      }
    release();
    if (info) info->status = QOP_SUCCESS;
    return 0;
  } catch (Fail &e) {
    release();
    fprintf(stderr, "QOPB_D3_sloppy_ddagd_batch: %s\n", e.msg.c_str());
    if (info) info->status = e.status;
    return -1;
  }
}
