// mixed.cuh -- storage formats, solver state and int16 hop building blocks
// shared by the reduced-precision solvers (mixed.cu: one system or several
// shifts of one system; batch.cu: several independent systems).
#pragma once
#include "qopb.h"
#include <cuda_fp16.h>

namespace qopb {

// ---------------------------------------------------------------- storage
// FP32 vector parity block: [3][Vh] float2
struct SpF32 {
  typedef float2 elem;
  static i64 block(i64 Vh) { return 3 * Vh; }
  static const char *name() { return "f32"; }
  static constexpr int site_bytes = 24;
  __device__ static void load(const float2 *b, int i, i64 Vh, float2 v[3]) {
    v[0] = b[i]; v[1] = b[Vh + i]; v[2] = b[2 * Vh + i];
  }
  __device__ static void store(float2 *b, int i, i64 Vh, float2 v[3]) {
    b[i] = v[0]; b[Vh + i] = v[1]; b[2 * Vh + i] = v[2];
  }
};

// FP16 vector parity block: [Vh] x 16 bytes = {half2 c0, c1, c2; float s}.
// Components are stored divided by the site's largest |re|,|im| (s), so
// every stored half lies in [-1, 1]; one 16-byte load per site.
struct SpF16 {
  typedef uint4 elem;
  static i64 block(i64 Vh) { return Vh; }
  static const char *name() { return "f16"; }
  static constexpr int site_bytes = 16;
  __device__ static void load(const uint4 *b, int i, i64, float2 v[3]) {
    uint4 u = b[i];
    float s = __uint_as_float(u.w);
    float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&u.x));
    float2 c = __half22float2(*reinterpret_cast<const __half2 *>(&u.y));
    float2 d = __half22float2(*reinterpret_cast<const __half2 *>(&u.z));
    v[0] = make_float2(a.x * s, a.y * s);
    v[1] = make_float2(c.x * s, c.y * s);
    v[2] = make_float2(d.x * s, d.y * s);
  }
  // stores the quantised site and returns the stored values in v
  __device__ static void store(uint4 *b, int i, i64, float2 v[3]) {
    float m = fmaxf(fmaxf(fmaxf(fabsf(v[0].x), fabsf(v[0].y)), fmaxf(fabsf(v[1].x), fabsf(v[1].y))),
                    fmaxf(fabsf(v[2].x), fabsf(v[2].y)));
    float inv = m > 0.f ? 1.0f / m : 0.f;
    __half2 h[3];
    uint4 u;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      h[c] = __floats2half2_rn(v[c].x * inv, v[c].y * inv);
      float2 f = __half22float2(h[c]);
      v[c] = make_float2(f.x * m, f.y * m);
    }
    u.x = *reinterpret_cast<unsigned *>(&h[0]);
    u.y = *reinterpret_cast<unsigned *>(&h[1]);
    u.z = *reinterpret_cast<unsigned *>(&h[2]);
    u.w = __float_as_uint(m);
    b[i] = u;
  }
};

// 16-bit fixed point: a component x is stored as u = q + 32768 with
// q = round(32767 x / s) in [-32767, 32767] and a float scale s per site
// (vectors) or per link (links): 15 bits of mantissa relative to the largest
// component.  Decoding needs no integer->float conversion: byte-permuting u
// under the exponent 0x4B gives the float 2^23 + u exactly, and subtracting
// 2^23 + 32768 gives q exactly; the scale is applied afterwards.
__device__ __forceinline__ float u16_lo(unsigned w) {
  return __int_as_float(__byte_perm(w, 0x4B000000u, 0x7610)) - 8421376.0f;
}
__device__ __forceinline__ float u16_hi(unsigned w) {
  return __int_as_float(__byte_perm(w, 0x4B000000u, 0x7632)) - 8421376.0f;
}
__device__ __forceinline__ unsigned u16_pack(float x, float y, float inv) {
  int a = __float2int_rn(x * inv), b = __float2int_rn(y * inv);
  a = max(-32767, min(32767, a)) + 32768;
  b = max(-32767, min(32767, b)) + 32768;
  return (unsigned)a | ((unsigned)b << 16);
}
__device__ __forceinline__ float absmax3(const float2 v[3]) {
  return fmaxf(fmaxf(fmaxf(fabsf(v[0].x), fabsf(v[0].y)), fmaxf(fabsf(v[1].x), fabsf(v[1].y))),
               fmaxf(fabsf(v[2].x), fabsf(v[2].y)));
}

// int16 vector parity block: [Vh] x 16 bytes = {u16 re/im x 3 colours; float s}
struct SpQ16 {
  typedef uint4 elem;
  static i64 block(i64 Vh) { return Vh; }
  static const char *name() { return "q16"; }
  static constexpr int site_bytes = 16;
  // integer-valued components and the factor c = s/32767 that scales them
  __device__ static float raw(uint4 u, float2 q[3]) {
    q[0] = make_float2(u16_lo(u.x), u16_hi(u.x));
    q[1] = make_float2(u16_lo(u.y), u16_hi(u.y));
    q[2] = make_float2(u16_lo(u.z), u16_hi(u.z));
    return __uint_as_float(u.w) * (1.0f / 32767.0f);
  }
  __device__ static void load(const uint4 *b, int i, i64, float2 v[3]) {
    const float c = raw(b[i], v);
#pragma unroll
    for (int k = 0; k < 3; k++) v[k] = make_float2(v[k].x * c, v[k].y * c);
  }
  __device__ static void store(uint4 *b, int i, i64, float2 v[3]) {
    const float m = absmax3(v);
    const float inv = m > 0.f ? 32767.0f / m : 0.f;
    uint4 u;
    u.x = u16_pack(v[0].x, v[0].y, inv);
    u.y = u16_pack(v[1].x, v[1].y, inv);
    u.z = u16_pack(v[2].x, v[2].y, inv);
    u.w = __float_as_uint(m);
    b[i] = u;
    load(&u, 0, 0, v);
  }
};

struct LinksSloppy { const void *a, *b, *c; };   // one parity

// int16 links, blocked for bulk copies: for every block of QB = 128 sites
// and every slot k, 5120 contiguous bytes = A[128] uint4 (elements 0-3),
// B[128] uint4 (elements 4-7), C[128] uint2 {element 8, float scale}; the
// slots of a block follow each other, so the links of 4 slots for 128 sites
// are one 20 KB contiguous span.  40 bytes per link.
constexpr int QB = 128;
constexpr int QSLOT = QB * 40;          // bytes per (block, slot)
struct LkQ16B {
  static const char *name() { return "q16"; }
  static constexpr int link_bytes = 40;
};
// FP32 links: a = [nl][9][Vh] float2
struct LkF32 {
  static const char *name() { return "f32"; }
  static constexpr int link_bytes = 72;
  __device__ static void load(const LinksSloppy &L, int k, int i, i64 Vh, float2 U[9]) {
    const float2 *p = (const float2 *)L.a + (i64)k * 9 * Vh + i;
#pragma unroll
    for (int e = 0; e < 9; e++) U[e] = p[e * Vh];
  }
};

// FP16 links: a = [nl][Vh] uint4 (e0..e3), b = [nl][Vh] uint4 (e4..e7),
// c = [nl][Vh] half2 (e8): 36 bytes per link in three coalesced loads
struct LkF16 {
  static const char *name() { return "f16"; }
  static constexpr int link_bytes = 36;
  __device__ static void unpack(uint4 u, float2 *U) {
    U[0] = __half22float2(*reinterpret_cast<const __half2 *>(&u.x));
    U[1] = __half22float2(*reinterpret_cast<const __half2 *>(&u.y));
    U[2] = __half22float2(*reinterpret_cast<const __half2 *>(&u.z));
    U[3] = __half22float2(*reinterpret_cast<const __half2 *>(&u.w));
  }
  __device__ static void load(const LinksSloppy &L, int k, int i, i64 Vh, float2 U[9]) {
    i64 o = (i64)k * Vh + i;
    unpack(((const uint4 *)L.a)[o], U);
    unpack(((const uint4 *)L.b)[o], U + 4);
    U[8] = __half22float2(((const __half2 *)L.c)[o]);
  }
};

// ---------------------------------------------------------------- state
enum { MIX_RUN = 0, MIX_UPDATE = 1, MIX_BREAK = 2 };
struct MixState {
  double rsq, rsq_old, alpha, beta, dp2, maxr2, stop, delta2, m2, red;
  int iter, max_iter, flag, tok;   // tok: iteration whose hop set alpha (fused update)
  double red3[3];
  int mbar_tries = -1;             // TMA-staged hops: polls per mbarrier wait (< 0: the default)
};

__device__ __forceinline__ void cfmaf(float2 &a, float2 u, float2 v) {
  a.x = fmaf(u.x, v.x, a.x); a.x = fmaf(-u.y, v.y, a.x);
  a.y = fmaf(u.x, v.y, a.y); a.y = fmaf(u.y, v.x, a.y);
}

// FP64 [3][Vh] parity block -> sloppy
template <class Sp>
__global__ void k_to_sloppy(typename Sp::elem *d, const double2 *s, i64 Vh) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Vh) return;
  float2 v[3];
#pragma unroll
  for (int c = 0; c < 3; c++) { double2 w = s[c * Vh + i]; v[c] = make_float2((float)w.x, (float)w.y); }
  Sp::store(d, i, Vh, v);
}

template <class T>
__global__ void k_copy_elems(T *d, const T *s, i64 n) {
  i64 k = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (k < n) d[k] = s[k];
}

// Long (Naik) links of asqtad and HISQ are c times a unitary matrix with one
// |c| for the whole lattice (naik/2 times products of U(3) links, times the
// +-1 phases).  With RECON they are stored as their first two rows divided by
// |c| (int16, no per-link scale) and the phase of det(L/|c|): 28 bytes
// A[128] uint4 (elements 0-3), B[128] uint2 (elements 4-5), C[128] float.
// The third row is det * conj(row0 x row1).  Fat links keep the 40-byte
// form.  In the blocked layout slots then alternate fat (5120 bytes per 128
// sites) and long (3584 bytes).
constexpr int QSLOTL = QB * 28;
__host__ __device__ constexpr int q16_slot_off(int k, bool recon) {
  return recon ? (k >> 1) * (QSLOT + QSLOTL) + (k & 1) * QSLOT : k * QSLOT;
}
__host__ __device__ constexpr int q16_block_bytes(int nl, bool recon) {
  return recon ? (nl / 2) * (QSLOT + QSLOTL) : nl * QSLOT;
}

enum { MIX_ERROR = 3 };

// neighbour of (x0..x3) = lex in parity p along mu by d, as a checkerboard index
struct NbrGeom { int L[4]; int str[4]; };
__device__ __forceinline__ int nbr_fast(const NbrGeom &n, const int x[4], int lex, int mu, int d) {
  int t = x[mu] + d;
  int off = d * n.str[mu];
  if (t >= n.L[mu]) off -= n.L[mu] * n.str[mu];
  else if (t < 0) off += n.L[mu] * n.str[mu];
  return (lex + off) >> 1;
}

// neighbour index with the direction chosen at run time (no indexed arrays)
__device__ __forceinline__ int nbr_sel(const NbrGeom &n, int x0, int x1, int x2, int x3, int lex, int mu, int d) {
  const int xm = mu == 0 ? x0 : mu == 1 ? x1 : mu == 2 ? x2 : x3;
  const int Lm = mu == 0 ? n.L[0] : mu == 1 ? n.L[1] : mu == 2 ? n.L[2] : n.L[3];
  const int sm = mu == 0 ? n.str[0] : mu == 1 ? n.str[1] : mu == 2 ? n.str[2] : n.str[3];
  const int t = xm + d;
  int off = d * sm;
  if (t >= Lm) off -= Lm * sm;
  else if (t < 0) off += Lm * sm;
  return (lex + off) >> 1;
}

// a += (link scale x site scale) x (integer link) (integer site): one slot
__device__ __forceinline__ void q16_slot(const uint4 ua, const uint4 ub, const uint2 uc, const uint4 nb, float2 a[3]) {
  float2 v[3];
  const float cv = SpQ16::raw(nb, v);
  const float sc = __uint_as_float(uc.y) * (1.0f / 32767.0f) * cv;
  float2 U[9];
  U[0] = make_float2(u16_lo(ua.x), u16_hi(ua.x)); U[1] = make_float2(u16_lo(ua.y), u16_hi(ua.y));
  U[2] = make_float2(u16_lo(ua.z), u16_hi(ua.z)); U[3] = make_float2(u16_lo(ua.w), u16_hi(ua.w));
  U[4] = make_float2(u16_lo(ub.x), u16_hi(ub.x)); U[5] = make_float2(u16_lo(ub.y), u16_hi(ub.y));
  U[6] = make_float2(u16_lo(ub.z), u16_hi(ub.z)); U[7] = make_float2(u16_lo(ub.w), u16_hi(ub.w));
  U[8] = make_float2(u16_lo(uc.x), u16_hi(uc.x));
#pragma unroll
  for (int r = 0; r < 3; r++) {
    float2 t = make_float2(0.f, 0.f);
    cfmaf(t, U[3 * r], v[0]);
    cfmaf(t, U[3 * r + 1], v[1]);
    cfmaf(t, U[3 * r + 2], v[2]);
    a[r].x = fmaf(sc, t.x, a[r].x);
    a[r].y = fmaf(sc, t.y, a[r].y);
  }
}

// one long slot stored as two rows + det phase: a += (|c|/32767 x site scale) U v
__device__ __forceinline__ void q16_slot_recon(const uint4 ua, const uint2 ub, const float phase, const uint4 nb,
                                               const float cl, float2 a[3]) {
  float2 v[3];
  const float cv = SpQ16::raw(nb, v);
  const float sc = cl * (1.0f / 32767.0f) * cv;
  float2 U[9];
  U[0] = make_float2(u16_lo(ua.x), u16_hi(ua.x)); U[1] = make_float2(u16_lo(ua.y), u16_hi(ua.y));
  U[2] = make_float2(u16_lo(ua.z), u16_hi(ua.z)); U[3] = make_float2(u16_lo(ua.w), u16_hi(ua.w));
  U[4] = make_float2(u16_lo(ub.x), u16_hi(ub.x)); U[5] = make_float2(u16_lo(ub.y), u16_hi(ub.y));
  float sn, cs;
  __sincosf(phase, &sn, &cs);
  const float2 z = make_float2(cs * (1.0f / 32767.0f), sn * (1.0f / 32767.0f));
  // row 2 = det * conj(row0 x row1), in units of the stored integers
  const float2 c0 = csub<float>(cmul<float>(U[1], U[5]), cmul<float>(U[2], U[4]));
  const float2 c1 = csub<float>(cmul<float>(U[2], U[3]), cmul<float>(U[0], U[5]));
  const float2 c2 = csub<float>(cmul<float>(U[0], U[4]), cmul<float>(U[1], U[3]));
  U[6] = cmul<float>(z, make_float2(c0.x, -c0.y));
  U[7] = cmul<float>(z, make_float2(c1.x, -c1.y));
  U[8] = cmul<float>(z, make_float2(c2.x, -c2.y));
#pragma unroll
  for (int r = 0; r < 3; r++) {
    float2 t = make_float2(0.f, 0.f);
    cfmaf(t, U[3 * r], v[0]);
    cfmaf(t, U[3 * r + 1], v[1]);
    cfmaf(t, U[3 * r + 2], v[2]);
    a[r].x = fmaf(sc, t.x, a[r].x);
    a[r].y = fmaf(sc, t.y, a[r].y);
  }
}

// Packed FP32x2 form of the two slot routines above (sm_100 f32x2 FMA):
// the link elements stay (re, im) pairs, the site's components enter
// pre-scaled and duplicated, and two packed accumulators per row collect
// t = sum U v.x and s = sum U v.y over all slots; the row is then
// (t.x - s.y, t.y + s.x) (q16_pk_rows).  About a third fewer instructions
// per slot than the scalar form; the rounding differs (the scale multiplies
// the site components before the link product).
__device__ __forceinline__ float2 u16_pair(unsigned w) {
  const float2 b = make_float2(__int_as_float(__byte_perm(w, 0x4B000000u, 0x7610)),
                               __int_as_float(__byte_perm(w, 0x4B000000u, 0x7632)));
  return __fadd2_rn(b, make_float2(-8421376.0f, -8421376.0f));
}

// site components times sc, duplicated: vx[c] = (re sc, re sc), vy[c] = (im sc, im sc).
// The integer pair comes out exact (u16_pair) and is scaled by one packed
// multiply, so each component carries a single rounding; folding the offset
// into an FMA instead (fma(2^23 + u, s, -(2^23 + 32768) s)) would round the
// offset product and add up to half a quantisation step per component.
__device__ __forceinline__ void q16_pk_site(const uint4 nb, float sc, float2 vx[3], float2 vy[3]) {
  const float s = sc * __uint_as_float(nb.w) * (1.0f / 32767.0f);
  const float2 s2 = make_float2(s, s);
  const unsigned w[3] = {nb.x, nb.y, nb.z};
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float2 v = __fmul2_rn(u16_pair(w[c]), s2);
    vx[c] = make_float2(v.x, v.x);
    vy[c] = make_float2(v.y, v.y);
  }
}

__device__ __forceinline__ void q16_pk_mul(const float2 U[9], const float2 vx[3], const float2 vy[3], float2 t[3],
                                           float2 s[3]) {
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      t[r] = __ffma2_rn(U[3 * r + c], vx[c], t[r]);
      s[r] = __ffma2_rn(U[3 * r + c], vy[c], s[r]);
    }
}

__device__ __forceinline__ void q16_slot_pk(const uint4 ua, const uint4 ub, const uint2 uc, const uint4 nb,
                                            float2 t[3], float2 s[3]) {
  float2 vx[3], vy[3];
  q16_pk_site(nb, __uint_as_float(uc.y) * (1.0f / 32767.0f), vx, vy);
  const float2 U[9] = {u16_pair(ua.x), u16_pair(ua.y), u16_pair(ua.z), u16_pair(ua.w), u16_pair(ub.x),
                       u16_pair(ub.y), u16_pair(ub.z), u16_pair(ub.w), u16_pair(uc.x)};
  q16_pk_mul(U, vx, vy, t, s);
}

// conj(a b - c d) of complex pairs
__device__ __forceinline__ float2 conj_cross(const float2 a, const float2 b, const float2 c, const float2 d) {
  float re = a.x * b.x;
  re = fmaf(-a.y, b.y, re);
  re = fmaf(-c.x, d.x, re);
  re = fmaf(c.y, d.y, re);
  float im = -(a.x * b.y);
  im = fmaf(-a.y, b.x, im);
  im = fmaf(c.x, d.y, im);
  im = fmaf(c.y, d.x, im);
  return make_float2(re, im);
}

// The third row never forms: row 2 = det conj(row0 x row1), so its product
// with the site is z sum_c conj(c_c) v_c (z = det / 32767), one complex dot
// folded into the row-2 accumulator after the phase.
__device__ __forceinline__ void q16_slot_recon_pk(const uint4 ua, const uint2 ub, const float phase, const uint4 nb,
                                                  const float cl, float2 t[3], float2 s[3]) {
  float2 vx[3], vy[3];
  q16_pk_site(nb, cl * (1.0f / 32767.0f), vx, vy);
  const float2 U[6] = {u16_pair(ua.x), u16_pair(ua.y), u16_pair(ua.z), u16_pair(ua.w), u16_pair(ub.x), u16_pair(ub.y)};
#pragma unroll
  for (int r = 0; r < 2; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      t[r] = __ffma2_rn(U[3 * r + c], vx[c], t[r]);
      s[r] = __ffma2_rn(U[3 * r + c], vy[c], s[r]);
    }
  const float2 k0 = conj_cross(U[1], U[5], U[2], U[4]);
  const float2 k1 = conj_cross(U[2], U[3], U[0], U[5]);
  const float2 k2 = conj_cross(U[0], U[4], U[1], U[3]);
  float2 tw = __fmul2_rn(k0, vx[0]), sw = __fmul2_rn(k0, vy[0]);
  tw = __ffma2_rn(k1, vx[1], tw);
  sw = __ffma2_rn(k1, vy[1], sw);
  tw = __ffma2_rn(k2, vx[2], tw);
  sw = __ffma2_rn(k2, vy[2], sw);
  const float2 w = make_float2(tw.x - sw.y, tw.y + sw.x);
  float sn, cs;
  __sincosf(phase, &sn, &cs);
  const float zx = cs * (1.0f / 32767.0f), zy = sn * (1.0f / 32767.0f);
  const float2 zw = make_float2(fmaf(zx, w.x, -zy * w.y), fmaf(zx, w.y, zy * w.x));
  t[2] = __fadd2_rn(t[2], zw);
}

__device__ __forceinline__ void q16_pk_rows(const float2 t[3], const float2 s[3], float2 a[3]) {
#pragma unroll
  for (int r = 0; r < 3; r++) a[r] = make_float2(t[r].x - s[r].y, t[r].y + s[r].x);
}

struct SloppyLinks {
  int nl = 0;
  void *a16 = nullptr, *b16 = nullptr, *c16 = nullptr;   // IEEE FP16 copy
  void *aq = nullptr;                                    // int16 fixed-point copy (blocked)
  int recon = 0;                                         // long links as 2 rows + det phase
  double c_long = 0;                                     // |c| of the long links when recon
  int recon_mode = -1;                                   // recon option the copy was built for
  FlaT<float> *f32 = nullptr;                            // FP32 copy
};

// link formats of the sloppy operator
enum { LK_F32 = 32, LK_Q16 = 16, LK_F16 = 15 };

// x += xs (FP64 += FP32), xs = 0 (mixed.cu)
__global__ void k_fold_x(double2 *x, float2 *xs, i64 n);

// reduced-precision copies of a link handle, built on first use (mixed.cu)
SloppyLinks *sloppy_get(FlaT<double> *f, int lkfmt);
LinksSloppy links_parity(SloppyLinks *s, int lkfmt, int p);

}  // namespace qopb
