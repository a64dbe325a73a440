// mixed.cu -- mixed-precision reliable-update CG for A = m^2 - D_eo D_oe
// (B200 addition; the reference's own mixed mode is the FP32 restart of
// lib/asqtad_invert_p.c:510-537, reproduced in solvers.cu).
//
// The Krylov iteration runs with FP16 (per-site scaled) or FP32 storage of
// links and vectors and FP32 arithmetic.  Everything that decides accuracy
// stays in FP64: all inner products are accumulated in double, the scalars
// alpha/beta/|r|^2 live in device memory as doubles, and whenever the
// iterated residual has dropped by `ru_delta` since the last update (or
// claims convergence) the solution is folded into an FP64 vector and the
// true residual b - A x is recomputed with the FP64 operator (Sleijpen-van
// der Vorst reliable update), replacing the sloppy residual; the search
// direction is kept, with beta recomputed from the true residual.
//
// One CG iteration is four launches with no host round trip:
//   K1  t  = D_oe p                     (sloppy hop, sum |t|^2)
//   K2  Ap = m^2 p - D_eo t             (sloppy hop, sum |p|^2 -> alpha)
//   K3  x += alpha p, r -= alpha Ap     (sum |r|^2 -> beta, update test)
//   K4  p  = r + beta p
// The last block of each reducing kernel writes the FP64 scalars; when K3
// requests a reliable update (or K2 detects breakdown) it sets a flag that
// turns every later launch of the chunk into a no-op.  The host launches
// `chunk` iterations at a time and only then reads the state.
#include "solvers.cuh"
#include "reduce.cuh"
#include "dslash.cuh"
#include "prof.cuh"
#include "fields.cuh"
#include "mixed.cuh"
#include "dd.cuh"
#include <algorithm>
#include <array>
#include <map>
#include <vector>
#include <cmath>

namespace qopb {

// KIND 1: out = D src (opposite parity of p);  KIND 2: out = m^2 same - D src
template <class Sp, class Lk, int NL, int KIND>
__global__ void __launch_bounds__(128)
k_mix_hop(typename Sp::elem *__restrict__ out, const typename Sp::elem *__restrict__ src, LinksSloppy lk,
          const typename Sp::elem *__restrict__ same, Geom g, int p, MixState *st, double *part, unsigned *count) {
  if (st->flag) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const i64 Vh = g.Vh;
  double acc1[1] = {0.0};
  if (i < Vh) {
    int x[4];
    site_coords(g, i, p, x);
    float2 a[3] = {make_float2(0, 0), make_float2(0, 0), make_float2(0, 0)};
#pragma unroll
    for (int k = 0; k < NL; k++) {
      const int j = nbr_index(g, x, slot_mu<NL>(k), slot_disp<NL>(k));
      float2 v[3], U[9];
      Sp::load(src, j, Vh, v);
      Lk::load(lk, k, i, Vh, U);
#pragma unroll
      for (int r = 0; r < 3; r++) {
        cfmaf(a[r], U[3 * r], v[0]);
        cfmaf(a[r], U[3 * r + 1], v[1]);
        cfmaf(a[r], U[3 * r + 2], v[2]);
      }
    }
    if (KIND == 1) {
      Sp::store(out, i, Vh, a);
      acc1[0] = (double)a[0].x * a[0].x + (double)a[0].y * a[0].y + (double)a[1].x * a[1].x +
                (double)a[1].y * a[1].y + (double)a[2].x * a[2].x + (double)a[2].y * a[2].y;
    } else {
      const float m2 = (float)st->m2;
      float2 s[3];
      Sp::load(same, i, Vh, s);
#pragma unroll
      for (int c = 0; c < 3; c++) a[c] = make_float2(m2 * s[c].x - a[c].x, m2 * s[c].y - a[c].y);
      Sp::store(out, i, Vh, a);
      acc1[0] = (double)s[0].x * s[0].x + (double)s[0].y * s[0].y + (double)s[1].x * s[1].x +
                (double)s[1].y * s[1].y + (double)s[2].x * s[2].x + (double)s[2].y * s[2].y;
    }
  }
  if (grid_sum<1>(acc1, part, count, &st->red)) {
    if (KIND == 1) {
      st->dp2 = st->red;
    } else {
      double pAp = st->dp2 + st->m2 * st->red;   // <p, A p> = |D p|^2 + m^2 |p|^2
      if (!(pAp > 0)) st->flag = MIX_BREAK;
      else st->alpha = st->rsq / pAp;
    }
  }
}

template <class Sp>
__global__ void __launch_bounds__(256)
k_mix_update(float2 *__restrict__ xs, typename Sp::elem *__restrict__ r, const typename Sp::elem *__restrict__ p,
             const typename Sp::elem *__restrict__ Ap, i64 Vh, MixState *st, double *part, unsigned *count) {
  if (st->flag) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc1[1] = {0.0};
  if (i < Vh) {
    const float al = (float)st->alpha;
    float2 pv[3], av[3], rv[3];
    Sp::load(p, i, Vh, pv);
    Sp::load(Ap, i, Vh, av);
    Sp::load(r, i, Vh, rv);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float2 xv = xs[c * Vh + i];
      xv.x = fmaf(al, pv[c].x, xv.x);
      xv.y = fmaf(al, pv[c].y, xv.y);
      xs[c * Vh + i] = xv;
      rv[c].x = fmaf(-al, av[c].x, rv[c].x);
      rv[c].y = fmaf(-al, av[c].y, rv[c].y);
    }
    Sp::store(r, i, Vh, rv);
    acc1[0] = (double)rv[0].x * rv[0].x + (double)rv[0].y * rv[0].y + (double)rv[1].x * rv[1].x +
              (double)rv[1].y * rv[1].y + (double)rv[2].x * rv[2].x + (double)rv[2].y * rv[2].y;
  }
  if (grid_sum<1>(acc1, part, count, &st->red)) {
    double rn = st->red;
    st->iter += 1;
    st->rsq_old = st->rsq;
    st->rsq = rn;
    st->beta = rn / st->rsq_old;
    if (rn > st->maxr2) st->maxr2 = rn;
    if (rn < st->delta2 * st->maxr2 || rn <= st->stop || st->iter >= st->max_iter) st->flag = MIX_UPDATE;
  }
}

template <class Sp>
__global__ void __launch_bounds__(256)
k_mix_p(typename Sp::elem *__restrict__ p, const typename Sp::elem *__restrict__ r, i64 Vh, MixState *st) {
  if (st->flag) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Vh) return;
  const float be = (float)st->beta;
  float2 pv[3], rv[3];
  Sp::load(p, i, Vh, pv);
  Sp::load(r, i, Vh, rv);
#pragma unroll
  for (int c = 0; c < 3; c++) pv[c] = make_float2(fmaf(be, pv[c].x, rv[c].x), fmaf(be, pv[c].y, rv[c].y));
  Sp::store(p, i, Vh, pv);
}

// Programmatic dependent launch (option pdl): a kernel launched with the
// attribute may be scheduled while the kernel ahead of it in the stream
// drains; griddepcontrol.wait holds it until that kernel has completed and
// its memory is visible.  Without the attribute the wait returns at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
static void launch_k(bool pdl, void (*k)(KArgs...), dim3 grid, dim3 block, cudaStream_t s, Args... args) {
  if (!pdl) {
    k<<<grid, block, 0, s>>>(args...);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  QCHECK(cudaLaunchKernelEx(&cfg, k, args...));
}

// x += alpha p, r -= alpha Ap and p = r + beta p in one pass (fused update:
// the scalars come from the KIND 3 hop).  Runs only for the iteration whose
// hop recorded `seq` in tok; when that hop set MIX_UPDATE, p is left to the
// reliable update, which recomputes beta from the true residual.
template <class Sp>
__global__ void __launch_bounds__(256)
k_mix_update_p(float2 *__restrict__ xs, typename Sp::elem *__restrict__ r, typename Sp::elem *__restrict__ p,
               const typename Sp::elem *__restrict__ Ap, i64 Vh, const MixState *st, int seq) {
  pdl_wait();
  if (st->tok != seq) return;
  const int fl = st->flag;
  if (fl != MIX_RUN && fl != MIX_UPDATE) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Vh) return;
  const float al = (float)st->alpha, be = (float)st->beta;
  float2 pv[3], av[3], rv[3];
  Sp::load(p, i, Vh, pv);
  Sp::load(Ap, i, Vh, av);
  Sp::load(r, i, Vh, rv);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    float2 xv = xs[c * Vh + i];
    xv.x = fmaf(al, pv[c].x, xv.x);
    xv.y = fmaf(al, pv[c].y, xv.y);
    xs[c * Vh + i] = xv;
    rv[c].x = fmaf(-al, av[c].x, rv[c].x);
    rv[c].y = fmaf(-al, av[c].y, rv[c].y);
  }
  Sp::store(r, i, Vh, rv);
  if (fl != MIX_RUN) return;
#pragma unroll
  for (int c = 0; c < 3; c++) pv[c] = make_float2(fmaf(be, pv[c].x, rv[c].x), fmaf(be, pv[c].y, rv[c].y));
  Sp::store(p, i, Vh, pv);
}

// ---------------------------------------------------------------- multi-shift
// Shifted systems (A + sigma_s) x_s = b ride on the base recursion with the
// multi-shift CG recurrences of lib/invert_cg_p.c:234-252 and :356-362:
//   zeta_{k+1} = zeta_k zeta_{k-1} alpha_{k-1} /
//                (alpha_k beta_{k-1} (zeta_{k-1} - zeta_k) + zeta_{k-1} alpha_{k-1} (1 + sigma alpha_k))
//   alpha_s = alpha_k zeta_{k+1} / zeta_k,   beta_s = beta_k zeta_{k+1} alpha_s / (zeta_k alpha_k)
//   x_s += alpha_s p_s,   p_s = zeta_{k+1} r + beta_s p_s
// (alpha = step length, beta = direction coefficient; alpha_{-1} = -1,
// beta_{-1} = 0, zeta_0 = zeta_{-1} = 1).  The scalars are FP64 in device
// memory; a shift stops being updated once zeta^2 |r|^2 is below its target.
constexpr int MS_MAX = 32;
struct MsShift {
  double sigma, z, zo, bo, stop;   // index 0 (base): bo = previous alpha
  double beo;                      // index 0 (base): previous beta (the fused update's recurrences)
  int active, pad;
};
struct MsVecs {
  void *p[MS_MAX];
  float2 *x[MS_MAX];
};

__device__ __forceinline__ void ms_step(const MsShift &s, double al, double be_old, double al_old, double &zn,
                                        double &as) {
  zn = s.z * s.zo * al_old;
  const double c1 = al * be_old * (s.zo - s.z) + s.zo * al_old * (1.0 + s.sigma * al);
  zn = c1 != 0.0 ? zn / c1 : 0.0;
  if (s.z != 0.0) as = al * zn / s.z;
  else zn = as = 0.0;
}

// base: x += alpha p, r -= alpha Ap, |r|^2; shifts: x_s += alpha_s p_s.
// Every block derives alpha_s from the state as it was at launch; the last
// block (after all others have read it) advances the recurrences in place.
template <class Sp>
__global__ void __launch_bounds__(256)
k_ms_update(float2 *__restrict__ xs, typename Sp::elem *__restrict__ r, const typename Sp::elem *__restrict__ p,
            const typename Sp::elem *__restrict__ Ap, i64 Vh, MixState *st, double *part, unsigned *count,
            MsShift *sh, int ns, MsVecs mv) {
  typedef typename Sp::elem E;
  if (st->flag) return;
  __shared__ float al_s[MS_MAX];
  const double al = st->alpha, be_old = st->beta, al_old = sh[0].bo;
  if (threadIdx.x < MS_MAX) {
    const int s = threadIdx.x;
    float v = 0.f;
    if (s > 0 && s < ns && sh[s].active) {
      double zn, as;
      ms_step(sh[s], al, be_old, al_old, zn, as);
      v = (float)as;
    }
    al_s[s] = v;
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc1[1] = {0.0};
  if (i < Vh) {
    const float alf = (float)al;
    float2 pv[3], av[3], rv[3];
    Sp::load(p, i, Vh, pv);
    Sp::load(Ap, i, Vh, av);
    Sp::load(r, i, Vh, rv);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float2 xv = xs[c * Vh + i];
      xv.x = fmaf(alf, pv[c].x, xv.x);
      xv.y = fmaf(alf, pv[c].y, xv.y);
      xs[c * Vh + i] = xv;
      rv[c].x = fmaf(-alf, av[c].x, rv[c].x);
      rv[c].y = fmaf(-alf, av[c].y, rv[c].y);
    }
    Sp::store(r, i, Vh, rv);
    acc1[0] = (double)rv[0].x * rv[0].x + (double)rv[0].y * rv[0].y + (double)rv[1].x * rv[1].x +
              (double)rv[1].y * rv[1].y + (double)rv[2].x * rv[2].x + (double)rv[2].y * rv[2].y;
    for (int s = 1; s < ns; s++) {
      const float a = al_s[s];
      if (a == 0.f) continue;
      float2 ps[3];
      Sp::load(reinterpret_cast<const E *>(mv.p[s]), i, Vh, ps);
      float2 *xp = mv.x[s];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        float2 xv = xp[c * Vh + i];
        xv.x = fmaf(a, ps[c].x, xv.x);
        xv.y = fmaf(a, ps[c].y, xv.y);
        xp[c * Vh + i] = xv;
      }
    }
  }
  if (grid_sum<1>(acc1, part, count, &st->red)) {
    const double rn = st->red;
    for (int s = 1; s < ns; s++) {
      MsShift &q = sh[s];
      if (!q.active) continue;
      double zn, as;
      ms_step(q, al, be_old, al_old, zn, as);
      q.zo = q.z;
      q.z = zn;
      q.bo = as;
      if (zn * zn * rn <= q.stop) q.active = 0;
    }
    sh[0].bo = al;
    st->iter += 1;
    st->rsq_old = st->rsq;
    st->rsq = rn;
    st->beta = rn / st->rsq_old;
    if (rn > st->maxr2) st->maxr2 = rn;
    if (rn < st->delta2 * st->maxr2 || rn <= st->stop || st->iter >= st->max_iter) st->flag = MIX_UPDATE;
  }
}

// p = r + beta p;  p_s = zeta_s r + beta_s p_s for the shifts still active
// (also records beta as the previous beta of the fused update's recurrences)
template <class Sp>
__global__ void __launch_bounds__(256)
k_ms_p(typename Sp::elem *__restrict__ p, const typename Sp::elem *__restrict__ r, i64 Vh, MixState *st,
       MsShift *sh, int ns, MsVecs mv) {
  typedef typename Sp::elem E;
  if (st->flag) return;
  __shared__ float pz[MS_MAX], pb[MS_MAX];
  const double be = st->beta, al = st->alpha;
  if (blockIdx.x == 0 && threadIdx.x == 0) sh[0].beo = be;   // no block reads sh[0] here
  if (threadIdx.x < MS_MAX) {
    const int s = threadIdx.x;
    float z = 0.f, b = 0.f;
    if (s > 0 && s < ns && sh[s].active) {
      const MsShift q = sh[s];
      const double d = q.zo * al;
      z = (float)q.z;
      b = d != 0.0 ? (float)(be * q.z * q.bo / d) : 0.f;
    }
    pz[s] = z;
    pb[s] = b;
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Vh) return;
  const float bef = (float)be;
  float2 pv[3], rv[3];
  Sp::load(p, i, Vh, pv);
  Sp::load(r, i, Vh, rv);
#pragma unroll
  for (int c = 0; c < 3; c++) pv[c] = make_float2(fmaf(bef, pv[c].x, rv[c].x), fmaf(bef, pv[c].y, rv[c].y));
  Sp::store(p, i, Vh, pv);
  for (int s = 1; s < ns; s++) {
    const float z = pz[s], b = pb[s];
    if (z == 0.f && b == 0.f) continue;
    E *q = reinterpret_cast<E *>(mv.p[s]);
    Sp::load(q, i, Vh, pv);
#pragma unroll
    for (int c = 0; c < 3; c++)
      pv[c] = make_float2(fmaf(b, pv[c].x, z * rv[c].x), fmaf(b, pv[c].y, z * rv[c].y));
    Sp::store(q, i, Vh, pv);
  }
}


// The multi-shift update after the fused-update hop (KIND 3), in one pass:
// base x += alpha p, r -= alpha Ap, p = r + beta p; every shift active at
// launch x_s += alpha_s p_s and p_s = zeta_{k+1} r + beta_s p_s.  alpha,
// beta and the new |r|^2 come from the hop; the shift scalars from the
// recurrences above (ms_step, and beta_s as in k_ms_p), derived in every
// block from the state at launch; the last block advances them and retires
// the shifts whose zeta^2 |r|^2 reached their target.  When the hop asked
// for a reliable update, p and the p_s are left to it (k_ms_p after the
// update, with beta recomputed).  Runs only for the iteration whose hop
// recorded `seq`.
template <class Sp>
__global__ void __launch_bounds__(256)
k_ms_update_fused(float2 *__restrict__ xs, typename Sp::elem *__restrict__ r, typename Sp::elem *__restrict__ p,
                  const typename Sp::elem *__restrict__ Ap, i64 Vh, MixState *st, int seq, double *part,
                  unsigned *count, MsShift *sh, int ns, MsVecs mv) {
  typedef typename Sp::elem E;
  pdl_wait();
  if (st->tok != seq) return;
  const int fl = st->flag;
  if (fl != MIX_RUN && fl != MIX_UPDATE) return;   // uniform: no block takes part in the ticket below
  __shared__ float al_s[MS_MAX], z_s[MS_MAX], b_s[MS_MAX];
  const double al = st->alpha, be = st->beta, rn = st->rsq, be_old = sh[0].beo, al_old = sh[0].bo;
  if (threadIdx.x < MS_MAX) {
    const int s = threadIdx.x;
    float a = 0.f, z = 0.f, b = 0.f;
    if (s > 0 && s < ns && sh[s].active) {
      double zn, as;
      ms_step(sh[s], al, be_old, al_old, zn, as);
      const double d = sh[s].z * al;
      a = (float)as;
      z = (float)zn;
      b = d != 0.0 ? (float)(be * zn * as / d) : 0.f;
    }
    al_s[s] = a;
    z_s[s] = z;
    b_s[s] = b;
  }
  __syncthreads();
  const bool run = fl == MIX_RUN;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < Vh) {
    const float alf = (float)al, bef = (float)be;
    float2 pv[3], av[3], rv[3];
    Sp::load(p, i, Vh, pv);
    Sp::load(Ap, i, Vh, av);
    Sp::load(r, i, Vh, rv);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float2 xv = xs[c * Vh + i];
      xv.x = fmaf(alf, pv[c].x, xv.x);
      xv.y = fmaf(alf, pv[c].y, xv.y);
      xs[c * Vh + i] = xv;
      rv[c].x = fmaf(-alf, av[c].x, rv[c].x);
      rv[c].y = fmaf(-alf, av[c].y, rv[c].y);
    }
    Sp::store(r, i, Vh, rv);
    if (run) {
#pragma unroll
      for (int c = 0; c < 3; c++) pv[c] = make_float2(fmaf(bef, pv[c].x, rv[c].x), fmaf(bef, pv[c].y, rv[c].y));
      Sp::store(p, i, Vh, pv);
    }
    for (int s = 1; s < ns; s++) {
      const float a = al_s[s];
      if (a == 0.f) continue;
      E *q = reinterpret_cast<E *>(mv.p[s]);
      float2 ps[3];
      Sp::load(q, i, Vh, ps);
      float2 *xp = mv.x[s];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        float2 xv = xp[c * Vh + i];
        xv.x = fmaf(a, ps[c].x, xv.x);
        xv.y = fmaf(a, ps[c].y, xv.y);
        xp[c * Vh + i] = xv;
      }
      if (!run) continue;
      const float z = z_s[s], b = b_s[s];
#pragma unroll
      for (int c = 0; c < 3; c++) ps[c] = make_float2(fmaf(b, ps[c].x, z * rv[c].x), fmaf(b, ps[c].y, z * rv[c].y));
      Sp::store(q, i, Vh, ps);
    }
  }
  double acc1[1] = {0.0};   // the reduction serves only to find the last block
  if (grid_sum<1>(acc1, part, count, &st->red)) {
    for (int s = 1; s < ns; s++) {
      MsShift &q = sh[s];
      if (!q.active) continue;
      double zn, as;
      ms_step(q, al, be_old, al_old, zn, as);
      q.zo = q.z;
      q.z = zn;
      q.bo = as;
      if (zn * zn * rn <= q.stop) q.active = 0;
    }
    sh[0].bo = al;
    sh[0].beo = be;
  }
}

// x += xs (FP64 += FP32), xs = 0
__global__ void k_fold_x(double2 *x, float2 *xs, i64 n) {
  i64 k = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (k >= n) return;
  float2 a = xs[k];
  double2 b = x[k];
  x[k] = make_double2(b.x + (double)a.x, b.y + (double)a.y);
  xs[k] = make_float2(0.f, 0.f);
}


// ---------------------------------------------------------------- sloppy links
__global__ void k_links_f16(uint4 *A, uint4 *B, __half2 *C, const double2 *src, int nl, i64 Vh) {
  i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;   // over [2][nl][Vh]
  if (s >= 2 * nl * Vh) return;
  i64 i = s % Vh, pk = s / Vh;    // pk = p*nl + k
  const double2 *b = src + pk * 9 * Vh + i;
  __half2 h[9];
#pragma unroll
  for (int e = 0; e < 9; e++) {
    double2 v = b[e * Vh];
    h[e] = __floats2half2_rn((float)v.x, (float)v.y);
  }
  uint4 u, w;
  u.x = *reinterpret_cast<unsigned *>(&h[0]); u.y = *reinterpret_cast<unsigned *>(&h[1]);
  u.z = *reinterpret_cast<unsigned *>(&h[2]); u.w = *reinterpret_cast<unsigned *>(&h[3]);
  w.x = *reinterpret_cast<unsigned *>(&h[4]); w.y = *reinterpret_cast<unsigned *>(&h[5]);
  w.z = *reinterpret_cast<unsigned *>(&h[6]); w.w = *reinterpret_cast<unsigned *>(&h[7]);
  A[s] = u;
  B[s] = w;
  C[s] = h[8];
}

// blocked int16 links: dst is [2 parities][nblk][nl slots][QSLOT bytes];
// sites beyond Vh in the last block are zero links

// largest unitarity defect |L L^+ / c^2 - 1| and the range of row-0 norms c
// over all long links; decides whether RECON is exact enough.  A grid of a
// few blocks per SM strides over the links; each block reduces its threads
// (warp shuffles, then its warps through shared memory) and one thread per
// block updates the three words (the values are non-negative, so their bit
// patterns order as integers).
__global__ void __launch_bounds__(256) k_long_check(const double2 *src, int nl, i64 Vh, unsigned long long *defect,
                                                    unsigned long long *cmax, unsigned long long *cmin) {
  const i64 n = 2 * (nl / 2) * Vh;   // over [2][nl/2 long slots][Vh]
  double d = 0, cx = 0, cn = 1e300;
  for (i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x; s < n; s += (i64)gridDim.x * blockDim.x) {
    const i64 i = s % Vh, r = s / Vh;
    const int k = 2 * (int)(r % (nl / 2)) + 1, p = (int)(r / (nl / 2));
    double2 e[9];
    for (int j = 0; j < 9; j++) e[j] = src[(((i64)p * nl + k) * 9 + j) * Vh + i];
    const double c2 = e[0].x * e[0].x + e[0].y * e[0].y + e[1].x * e[1].x + e[1].y * e[1].y + e[2].x * e[2].x +
                      e[2].y * e[2].y;
    const double ic2 = 1.0 / c2;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) {
        double re = 0, im = 0;
        for (int j = 0; j < 3; j++) {
          double2 x = e[3 * a + j], y = e[3 * b + j];
          re += x.x * y.x + x.y * y.y;
          im += x.y * y.x - x.x * y.y;
        }
        re = re * ic2 - (a == b ? 1.0 : 0.0);
        im = im * ic2;
        d = fmax(d, fmax(fabs(re), fabs(im)));
      }
    const double c = sqrt(c2);
    cx = fmax(cx, c);
    cn = fmin(cn, c);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    d = fmax(d, __shfl_xor_sync(0xffffffffu, d, o));
    cx = fmax(cx, __shfl_xor_sync(0xffffffffu, cx, o));
    cn = fmin(cn, __shfl_xor_sync(0xffffffffu, cn, o));
  }
  __shared__ double sd[8], sx[8], sn[8];
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { sd[w] = d; sx[w] = cx; sn[w] = cn; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); k++) {
      d = fmax(d, sd[k]);
      cx = fmax(cx, sx[k]);
      cn = fmin(cn, sn[k]);
    }
    atomicMax(defect, (unsigned long long)__double_as_longlong(d));
    atomicMax(cmax, (unsigned long long)__double_as_longlong(cx));
    atomicMin(cmin, (unsigned long long)__double_as_longlong(cn));
  }
}

__global__ void k_links_q16b(unsigned char *dst, const double2 *src, int nl, i64 Vh, i64 nblk, int recon,
                             double c_long) {
  i64 s = blockIdx.x * (i64)blockDim.x + threadIdx.x;   // over [2][nblk][nl][QB]
  if (s >= 2 * nblk * nl * QB) return;
  const int t = (int)(s % QB);
  const i64 r = s / QB;
  const int k = (int)(r % nl);
  const i64 pb = r / nl, b = pb % nblk, p = pb / nblk;
  const i64 i = b * QB + t;
  unsigned char *blk = dst + (size_t)pb * q16_block_bytes(nl, recon != 0);
  if (recon && (k & 1)) {
    double2 e[9];
    for (int j = 0; j < 9; j++)
      e[j] = i < Vh ? src[((p * nl + k) * 9 + j) * Vh + i] : make_double2(j % 4 == 0 ? c_long : 0.0, 0.0);
    const double2 d = cadd<double>(
        csub<double>(cmul<double>(e[0], csub<double>(cmul<double>(e[4], e[8]), cmul<double>(e[5], e[7]))),
                     cmul<double>(e[1], csub<double>(cmul<double>(e[3], e[8]), cmul<double>(e[5], e[6])))),
        cmul<double>(e[2], csub<double>(cmul<double>(e[3], e[7]), cmul<double>(e[4], e[6]))));
    const float phase = (float)atan2(d.y, d.x);   // arg det(L/|c|) = arg det(L)
    const float inv = (float)(32767.0 / c_long);
    float2 f[6];
    for (int j = 0; j < 6; j++) f[j] = make_float2((float)e[j].x, (float)e[j].y);
    unsigned char *base = blk + q16_slot_off(k, true);
    reinterpret_cast<uint4 *>(base)[t] =
        make_uint4(u16_pack(f[0].x, f[0].y, inv), u16_pack(f[1].x, f[1].y, inv), u16_pack(f[2].x, f[2].y, inv),
                   u16_pack(f[3].x, f[3].y, inv));
    reinterpret_cast<uint2 *>(base + 16 * QB)[t] = make_uint2(u16_pack(f[4].x, f[4].y, inv), u16_pack(f[5].x, f[5].y, inv));
    reinterpret_cast<float *>(base + 24 * QB)[t] = phase;
    return;
  }
  float2 e[9];
  float m = 0.f;
#pragma unroll
  for (int j = 0; j < 9; j++) {
    e[j] = make_float2(0.f, 0.f);
    if (i < Vh) {
      double2 v = src[((p * nl + k) * 9 + j) * Vh + i];
      e[j] = make_float2((float)v.x, (float)v.y);
    }
    m = fmaxf(m, fmaxf(fabsf(e[j].x), fabsf(e[j].y)));
  }
  const float inv = m > 0.f ? 32767.0f / m : 0.f;
  unsigned char *base = blk + q16_slot_off(k, recon != 0);
  reinterpret_cast<uint4 *>(base)[t] =
      make_uint4(u16_pack(e[0].x, e[0].y, inv), u16_pack(e[1].x, e[1].y, inv), u16_pack(e[2].x, e[2].y, inv),
                 u16_pack(e[3].x, e[3].y, inv));
  reinterpret_cast<uint4 *>(base + 16 * QB)[t] =
      make_uint4(u16_pack(e[4].x, e[4].y, inv), u16_pack(e[5].x, e[5].y, inv), u16_pack(e[6].x, e[6].y, inv),
                 u16_pack(e[7].x, e[7].y, inv));
  reinterpret_cast<uint2 *>(base + 32 * QB)[t] = make_uint2(u16_pack(e[8].x, e[8].y, inv), __float_as_uint(m));
}

// ---------------------------------------------------------------- TMA-staged hop
// Variant 1 (TMA): link data of GRP slots x 128 sites (GRP x 5 KB,
// contiguous in the blocked layout) is fetched by one cp.async.bulk into
// shared memory against an mbarrier; two buffers alternate so the next
// group's links stream in while the current group is computed.  Neighbour
// sites are read with ordinary loads (L1/L2 hits) issued before the group's
// barrier wait.  Every wait is bounded: on timeout the kernel raises
// MIX_ERROR and skips the work.
// Variant 2 (LDG): the same blocked layout read with plain coalesced loads,
// the raw words of BATCH slots loaded before any of them is decoded so that
// BATCH x 56 bytes per thread are in flight.

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, unsigned phase) {
  unsigned ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok) : "r"(smem_u32(bar)), "r"(phase) : "memory");
  return ok != 0;
}
// non-blocking probe of the phase (mbarrier.test_wait never suspends)
__device__ __forceinline__ bool mbar_test(uint64_t *bar, unsigned phase) {
  unsigned ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok) : "r"(smem_u32(bar)), "r"(phase) : "memory");
  return ok != 0;
}
// a bounded wait: false after `tries` polls (the caller raises MIX_ERROR).
// The default limit polls with try_wait (which may suspend the thread for a
// while per poll); a limit of 16 polls or fewer (option mbar_tries) polls
// with the non-blocking test_wait, so that a short limit really is short,
// and a limit of 0 gives up at once
constexpr int MBAR_TRIES = 1 << 22;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned phase, int tries = MBAR_TRIES) {
  if (tries <= 16) {
    for (int it = 0; it < tries; it++)
      if (mbar_test(bar, phase)) return true;
    return false;
  }
  for (int it = 0; it < tries; it++)
    if (mbar_try(bar, phase)) return true;
  return false;
}


// KIND epilogue shared by both variants; returns the value to reduce
template <int KIND>
__device__ __forceinline__ double q16_epilogue(uint4 *out, const uint4 *same, int i, i64 Vh, float m2, float2 a[3]) {
  if (KIND == 1) {
    SpQ16::store(out, i, Vh, a);
    return (double)a[0].x * a[0].x + (double)a[0].y * a[0].y + (double)a[1].x * a[1].x + (double)a[1].y * a[1].y +
           (double)a[2].x * a[2].x + (double)a[2].y * a[2].y;
  }
  float2 sv[3];
  SpQ16::load(same, i, Vh, sv);
#pragma unroll
  for (int c = 0; c < 3; c++) a[c] = make_float2(m2 * sv[c].x - a[c].x, m2 * sv[c].y - a[c].y);
  SpQ16::store(out, i, Vh, a);
  return (double)sv[0].x * sv[0].x + (double)sv[0].y * sv[0].y + (double)sv[1].x * sv[1].x +
         (double)sv[1].y * sv[1].y + (double)sv[2].x * sv[2].x + (double)sv[2].y * sv[2].y;
}

template <int KIND>
__device__ __forceinline__ void q16_finish(double (&acc1)[1], double *part, unsigned *count, MixState *st) {
  if (grid_sum<1>(acc1, part, count, &st->red)) {
    if (KIND == 1) {
      st->dp2 = st->red;
    } else if (st->flag != MIX_ERROR) {
      double pAp = st->dp2 + st->m2 * st->red;   // <p, A p> = |D p|^2 + m^2 |p|^2
      if (!(pAp > 0)) st->flag = MIX_BREAK;
      else st->alpha = st->rsq / pAp;
    }
  }
}

// KIND 3 (fused update): the KIND 2 hop that also reduces <r, Ap> and
// |Ap|^2, so that its last block knows alpha, the new |r|^2 =
// |r|^2 - 2 alpha <r, Ap> + alpha^2 |Ap|^2 and beta before the update runs
__device__ __forceinline__ void q16_epilogue3(uint4 *out, const uint4 *same, const uint4 *rres, int i, i64 Vh,
                                              float m2, float2 a[3], double (&acc)[3]) {
  acc[0] += q16_epilogue<2>(out, same, i, Vh, m2, a);   // a becomes Ap
  float2 rv[3];
  SpQ16::load(rres, i, Vh, rv);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    acc[1] += (double)rv[c].x * a[c].x + (double)rv[c].y * a[c].y;
    acc[2] += (double)a[c].x * a[c].x + (double)a[c].y * a[c].y;
  }
}

// alpha, the new |r|^2, beta and the reliable-update test from the sums in
// dp2 and red3 (one thread)
__device__ __forceinline__ void mix_scalars3(MixState *st, int seq) {
  {
    if (st->flag != MIX_RUN) return;
    const double pAp = st->dp2 + st->m2 * st->red3[0];
    if (!(pAp > 0)) { st->flag = MIX_BREAK; return; }
    const double al = st->rsq / pAp;
    const double rn = st->rsq - 2.0 * al * st->red3[1] + al * al * st->red3[2];
    st->alpha = al;
    st->iter += 1;
    st->rsq_old = st->rsq;
    st->rsq = rn;
    st->beta = rn / st->rsq_old;
    if (rn > st->maxr2) st->maxr2 = rn;
    st->tok = seq;
    if (!(rn > 0) || rn < st->delta2 * st->maxr2 || rn <= st->stop || st->iter >= st->max_iter) st->flag = MIX_UPDATE;
  }
}

// DDQ (decomposed lattice): the sums are summed over the processes first,
// so the scalars come from k_mix_scalars3 after the all-reduce
template <bool DDQ>
__device__ __forceinline__ void q16_finish3(double (&acc)[3], double *part, unsigned *count, MixState *st, int seq) {
  if (grid_sum<3>(acc, part, count, st->red3) && !DDQ) mix_scalars3(st, seq);
}

__global__ void k_mix_scalars3(MixState *st, int seq) { mix_scalars3(st, seq); }

template <int NL, int KIND, int GRP>
__global__ void __launch_bounds__(QB)
k_mix_hop_q16(uint4 *__restrict__ out, const uint4 *__restrict__ src, const unsigned char *__restrict__ lk,
              const uint4 *__restrict__ same, Geom g, NbrGeom ng, int p, MixState *st, double *part,
              unsigned *count) {
  if (st->flag) return;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];
  constexpr int NG = NL / GRP;
  constexpr int GB = GRP * QSLOT;
  const int tid = threadIdx.x;
  const i64 Vh = g.Vh;
  const int i = blockIdx.x * QB + tid;
  const unsigned char *gl = lk + (size_t)blockIdx.x * NL * QSLOT;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
#pragma unroll
    for (int gi = 0; gi < 2 && gi < NG; gi++) {
      mbar_expect_tx(&bar[gi], GB);
      bulk_g2s(smem + gi * GB, gl + gi * GB, GB, &bar[gi]);
    }
  }
  const bool live = i < Vh;
  int x[4] = {0, 0, 0, 0}, lex = 0;
  if (live) {
    site_coords(g, i, p, x);
    lex = ((x[0] * g.L[1] + x[1]) * g.L[2] + x[2]) * g.L[3] + x[3];
  }
  float2 a[3] = {make_float2(0, 0), make_float2(0, 0), make_float2(0, 0)};
  bool ok = true;
  const int tries = st->mbar_tries >= 0 ? st->mbar_tries : MBAR_TRIES;
  int issued[2] = {NG > 0 ? 1 : 0, NG > 1 ? 1 : 0}, waited[2] = {0, 0};   // thread 0 bookkeeping
#pragma unroll
  for (int gi = 0; gi < NG; gi++) {
    const int buf = gi & 1;
    uint4 nb[GRP];
#pragma unroll
    for (int s = 0; s < GRP; s++) {
      const int k = gi * GRP + s;
      nb[s] = live ? src[nbr_fast(ng, x, lex, slot_mu<NL>(k), slot_disp<NL>(k))] : make_uint4(0, 0, 0, 0);
    }
    const bool arrived = mbar_wait_bounded(&bar[buf], (gi >> 1) & 1, tries);
    if (!arrived) ok = false;
    else waited[buf]++;
    if (arrived && live) {
      const unsigned char *sb = smem + buf * GB;
#pragma unroll
      for (int s = 0; s < GRP; s++) {
        const unsigned char *ls = sb + s * QSLOT;
        q16_slot(reinterpret_cast<const uint4 *>(ls)[tid], reinterpret_cast<const uint4 *>(ls + 16 * QB)[tid],
                 reinterpret_cast<const uint2 *>(ls + 32 * QB)[tid], nb[s], a);
      }
    }
    if (gi + 2 < NG) {
      __syncthreads();                 // every thread is done with this buffer
      if (tid == 0 && ok) {
        mbar_expect_tx(&bar[buf], GB);
        bulk_g2s(smem + buf * GB, gl + (gi + 2) * GB, GB, &bar[buf]);
        issued[buf]++;
      }
    }
  }
  if (!ok) {
    st->flag = MIX_ERROR;
    if (tid == 0)   // let copies still in flight land before the block exits (bounded, default limit)
      for (int b2 = 0; b2 < 2; b2++)
        while (waited[b2] < issued[b2] && mbar_wait_bounded(&bar[b2], waited[b2] & 1)) waited[b2]++;
  }
  double acc1[1] = {0.0};
  if (live) acc1[0] = q16_epilogue<KIND>(out, same, i, Vh, (float)st->m2, a);
  q16_finish<KIND>(acc1, part, count, st);
}


// ---------------------------------------------------------------- cp.async-pipelined hop
// Variants 17-19: persistent grid; every thread streams the raw words of its
// next R slots (the link and the neighbour site) into its own ring in shared
// memory with cp.async, so R x 56 bytes per thread are in flight without
// holding registers.  Slots are consumed in order across site blocks (the
// first slots of the next site block are fetched while the current block's
// last ones are computed).  The ring has R + 1 stages and a stage is refilled
// one slot after it was read.  Only the thread that wrote a stage reads it,
// so cp.async.wait_group alone orders the data: no barrier.  Sites beyond Vh
// in the last block fetch their (zero) padding links and site 0's
// neighbours, and are not stored.
__device__ __forceinline__ void cpa16(void *sm, const void *gm) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sm)), "l"(gm) : "memory");
}
__device__ __forceinline__ void cpa8(void *sm, const void *gm) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(sm)), "l"(gm) : "memory");
}
__device__ __forceinline__ void cpa4(void *sm, const void *gm) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(sm)), "l"(gm) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cpa_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int NL, int KIND, bool RECON, int R, int MINB>
__global__ void __launch_bounds__(QB, MINB)
k_mix_hop_q16a(uint4 *__restrict__ out, const uint4 *__restrict__ src, const unsigned char *__restrict__ lk,
               const uint4 *__restrict__ same, Geom g, NbrGeom ng, int p, MixState *st, double *part,
               unsigned *count, float c_long) {
  if (st->flag) return;
  constexpr int S = R + 1;
  __shared__ __align__(16) uint4 sa[S][QB];
  __shared__ __align__(16) uint4 sb[S][QB];
  __shared__ __align__(16) uint4 sn[S][QB];
  __shared__ __align__(16) uint2 sc[S][QB];
  const int tid = threadIdx.x;
  const i64 Vh = g.Vh;
  const int nsb = (int)((Vh + QB - 1) / QB);
  // issue cursor: site block, slot, this thread's site coordinates there
  int isb = blockIdx.x, ik = 0, ilex = 0, is = 0;
  int y0 = 0, y1 = 0, y2 = 0, y3 = 0;
  auto site_of = [&](int blk) {
    const i64 i = (i64)blk * QB + tid;
    int x[4];
    site_coords(g, i < Vh ? (int)i : 0, p, x);
    y0 = x[0]; y1 = x[1]; y2 = x[2]; y3 = x[3];
    ilex = ((y0 * g.L[1] + y1) * g.L[2] + y2) * g.L[3] + y3;
  };
  auto issue = [&]() {
    if (isb < nsb) {
      const unsigned char *ls = lk + (size_t)isb * q16_block_bytes(NL, RECON) + q16_slot_off(ik, RECON);
      if (RECON && (ik & 1)) {
        cpa16(&sa[is][tid], ls + 16 * tid);
        cpa8(&sb[is][tid], ls + 16 * QB + 8 * tid);
        cpa4(&sc[is][tid], ls + 24 * QB + 4 * tid);
      } else {
        cpa16(&sa[is][tid], ls + 16 * tid);
        cpa16(&sb[is][tid], ls + 16 * QB + 16 * tid);
        cpa8(&sc[is][tid], ls + 32 * QB + 8 * tid);
      }
      const int j = nbr_sel(ng, y0, y1, y2, y3, ilex, slot_mu<NL>(ik), slot_disp<NL>(ik));
      cpa16(&sn[is][tid], src + j);
      if (++ik == NL) {
        ik = 0;
        isb += gridDim.x;
        if (isb < nsb) site_of(isb);
      }
    }
    cpa_commit();
    is = (is + 1 == S) ? 0 : is + 1;
  };
  if (isb < nsb) site_of(isb);
#pragma unroll
  for (int r = 0; r < R; r++) issue();
  int cs = 0;   // stage being consumed
  double acc1[1] = {0.0};
  for (int cb = blockIdx.x; cb < nsb; cb += gridDim.x) {
    const int i = cb * QB + tid;
    float2 a[3] = {make_float2(0, 0), make_float2(0, 0), make_float2(0, 0)};
#pragma unroll
    for (int k = 0; k < NL; k++) {
      cpa_wait<R - 1>();
      const uint4 ua = sa[cs][tid], nb = sn[cs][tid];
      if (RECON && (k & 1)) {
        const uint4 w = sb[cs][tid];
        const uint2 c = sc[cs][tid];
        q16_slot_recon(ua, make_uint2(w.x, w.y), __uint_as_float(c.x), nb, c_long, a);
      } else {
        q16_slot(ua, sb[cs][tid], sc[cs][tid], nb, a);
      }
      cs = (cs + 1 == S) ? 0 : cs + 1;
      issue();   // refills the stage read one slot ago
    }
    if (i < Vh) acc1[0] += q16_epilogue<KIND>(out, same, i, Vh, (float)st->m2, a);
  }
  cpa_wait<0>();
  q16_finish<KIND>(acc1, part, count, st);
}

// PERSIST: a grid of (SMs x MINB) blocks strides over the site blocks, so
// no partial last wave of blocks leaves SMs idle
// PK: packed FP32x2 arithmetic (q16_slot_pk).  DDQ (with PK, decomposed
// lattice): a neighbour outside the block comes from the halos of gh (an
// up record multiplies the link as usual; a down record is the product
// -U^+ psi and is added as is)
// PF > 0 (persistent variants 29-31): thread 0 of a block asks L2 to fetch
// the link bytes of the slot batch PF batches ahead of the one the block
// starts (cp.async.bulk.prefetch.L2: no destination, no registers, no
// completion to wait for), so the block's own loads of that batch later hit
// L2 instead of waiting on HBM.  Batch b of site block sb is the contiguous
// span of slots [b BATCH, (b + 1) BATCH) of that block's link record.
__device__ __forceinline__ void l2_prefetch_bulk(const void *p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

template <int NL, int KIND, int BATCH, bool RECON, int MINB = 1, bool PERSIST = false, bool PK = false,
          bool DDQ = false, int PF = 0>
__global__ void __launch_bounds__(QB, MINB)
k_mix_hop_q16r(uint4 *__restrict__ out, const uint4 *__restrict__ src, const unsigned char *__restrict__ lk,
               const uint4 *__restrict__ same, Geom g, NbrGeom ng, int p, MixState *st, double *part,
               unsigned *count, float c_long, const uint4 *__restrict__ rres = nullptr, int seq = 0,
               DdQ16Ghost gh = DdQ16Ghost()) {
  if constexpr (PK) pdl_wait();   // the packed variants may be launched as dependents
  if (st->flag) return;
  const int tid = threadIdx.x;
  const i64 Vh = g.Vh;
  const int nsb = PERSIST ? (int)((Vh + QB - 1) / QB) : 0;
  double acc1[KIND == 3 ? 3 : 1];
#pragma unroll
  for (int k = 0; k < (KIND == 3 ? 3 : 1); k++) acc1[k] = 0.0;
  int sb = blockIdx.x;
  do {
  const int i = sb * QB + tid;
  const unsigned char *gl = lk + (size_t)sb * q16_block_bytes(NL, RECON);
  if (i < Vh) {
    int x[4];
    site_coords(g, i, p, x);
    const int lex = ((x[0] * g.L[1] + x[1]) * g.L[2] + x[2]) * g.L[3] + x[3];
    float2 a[3] = {make_float2(0, 0), make_float2(0, 0), make_float2(0, 0)};
    float2 pt[3] = {make_float2(0, 0), make_float2(0, 0), make_float2(0, 0)}, ps[3] = {pt[0], pt[1], pt[2]};
    // halo face index per decomposed direction: one per site, shared by the
    // four slots of that direction
    int hfi[4] = {0, 0, 0, 0};
    if constexpr (DDQ) {
#pragma unroll
      for (int mu = 0; mu < 4; mu++)
        if (gh.mask >> mu & 1) hfi[mu] = dd_face_index(g, x, mu);
    }
#pragma unroll
    for (int k0 = 0; k0 < NL; k0 += BATCH) {
      if constexpr (PERSIST && PF > 0) {
        constexpr int NB = NL / BATCH;
        if (tid == 0) {
          const int lin = k0 / BATCH + PF, blk = sb + (lin / NB) * gridDim.x, bb = lin % NB;
          if (blk < nsb) {
            const int o0 = q16_slot_off(bb * BATCH, RECON), o1 = q16_slot_off((bb + 1) * BATCH, RECON);
            l2_prefetch_bulk(lk + (size_t)blk * q16_block_bytes(NL, RECON) + o0, (unsigned)(o1 - o0));
          }
        }
      }
      uint4 ua[BATCH], ub[BATCH], nb[BATCH];
      uint2 uc[BATCH];
      bool prd[BATCH];
#pragma unroll
      for (int s = 0; s < BATCH; s++) {
        const int k = k0 + s;
        prd[s] = false;
        const unsigned char *ls = gl + q16_slot_off(k, RECON);
        ua[s] = __ldcs(reinterpret_cast<const uint4 *>(ls) + tid);
        if (RECON && (k & 1)) {
          uint2 w = __ldcs(reinterpret_cast<const uint2 *>(ls + 16 * QB) + tid);
          ub[s] = make_uint4(w.x, w.y, 0u, 0u);
          uc[s] = make_uint2(__float_as_uint(__ldcs(reinterpret_cast<const float *>(ls + 24 * QB) + tid)), 0u);
        } else {
          ub[s] = __ldcs(reinterpret_cast<const uint4 *>(ls + 16 * QB) + tid);
          uc[s] = __ldcs(reinterpret_cast<const uint2 *>(ls + 32 * QB) + tid);
        }
        const int mu = slot_mu<NL>(k), dsp = slot_disp<NL>(k);
        const uint4 *np = src + nbr_fast(ng, x, lex, mu, dsp);
        if (DDQ && (gh.mask >> mu & 1)) {   // uniform over the launch: no divergence here
          // the halo address is selected, not branched to: every lane issues
          // one load per slot (each warp of a split x3 row has boundary lanes)
          const int y = x[mu] + dsp, fh = gh.fh[mu], fi = hfi[mu];
          const bool cross = (unsigned)y >= (unsigned)g.L[mu];
          const int sl = max(dd_halo_slab(g.L[mu], y, dsp), 0);   // in range when unused
          const uint4 *hp = (y < 0 ? gh.dn[mu] : gh.up[mu]) + (i64)sl * fh + fi;
          np = cross ? hp : np;
          prd[s] = cross && y < 0;
        }
        nb[s] = *np;
      }
#pragma unroll
      for (int s = 0; s < BATCH; s++) {
        if (DDQ && prd[s]) {   // a = (t.x - s.y, t.y + s.x): the product enters t
          float2 z[3];
          SpQ16::load(&nb[s], 0, 0, z);
#pragma unroll
          for (int r = 0; r < 3; r++) { pt[r].x += z[r].x; pt[r].y += z[r].y; }
          continue;
        }
        if (PK) {
          if (RECON && ((k0 + s) & 1))
            q16_slot_recon_pk(ua[s], make_uint2(ub[s].x, ub[s].y), __uint_as_float(uc[s].x), nb[s], c_long, pt, ps);
          else
            q16_slot_pk(ua[s], ub[s], uc[s], nb[s], pt, ps);
        } else if (RECON && ((k0 + s) & 1)) {
          q16_slot_recon(ua[s], make_uint2(ub[s].x, ub[s].y), __uint_as_float(uc[s].x), nb[s], c_long, a);
        } else {
          q16_slot(ua[s], ub[s], uc[s], nb[s], a);
        }
      }
    }
    if (PK) q16_pk_rows(pt, ps, a);
    if constexpr (KIND == 3) q16_epilogue3(out, same, rres, i, Vh, (float)st->m2, a, acc1);
    else acc1[0] += q16_epilogue<KIND>(out, same, i, Vh, (float)st->m2, a);
  }
  } while (PERSIST && (sb += gridDim.x) < nsb);
  if constexpr (KIND == 3) q16_finish3<DDQ>(acc1, part, count, st, seq);
  else q16_finish<KIND>(acc1, part, count, st);
}


static std::map<void *, SloppyLinks *> g_sloppy;

void sloppy_invalidate(void *fla_any) {
  auto it = g_sloppy.find(fla_any);
  if (it == g_sloppy.end()) return;
  SloppyLinks *s = it->second;
  if (s->a16) { dfree(s->a16); dfree(s->b16); dfree(s->c16); }
  if (s->aq) dfree(s->aq);
  if (s->f32) fla_destroy<float>(s->f32);
  delete s;
  g_sloppy.erase(it);
}


SloppyLinks *sloppy_get(FlaT<double> *f, int lkfmt) {
  SloppyLinks *&s = g_sloppy[(void *)f];
  if (!s) { s = new SloppyLinks(); s->nl = f->nlinks; }
  const Geom &g = ctx().g;
  const i64 n = 2LL * f->nlinks * g.Vh;
  if (lkfmt == LK_F16 && !s->a16) {
    s->a16 = dmalloc(sizeof(uint4) * n);
    s->b16 = dmalloc(sizeof(uint4) * n);
    s->c16 = dmalloc(sizeof(__half2) * n);
    k_links_f16<<<grid_for(n, 256), 256, 0, ctx().s>>>((uint4 *)s->a16, (uint4 *)s->b16, (__half2 *)s->c16, f->d,
                                                       f->nlinks, g.Vh);
    QLAUNCH();
  }
  // the TMA variants need equal slot sizes: reconstruction only with the
  // plain-load kernels, and only if the long links pass the unitarity check
  const int want_recon = (ctx().opt.recon_long && ctx().opt.hop_kernel != 1 && ctx().opt.hop_kernel != 2) ? 1 : 0;
  if (lkfmt == LK_Q16 && s->aq && s->recon_mode != want_recon) { dfree(s->aq); s->aq = nullptr; }
  if (lkfmt == LK_Q16 && !s->aq) {
    const i64 nblk = (g.Vh + QB - 1) / QB;
    int recon = 0;
    double c_long = 0;
    if (want_recon && f->nlinks == 16) {
      unsigned long long *st = dalloc<unsigned long long>(3);
      unsigned long long init[3] = {0ull, 0ull, 0ull};
      const double big = 1e300;
      memcpy(&init[2], &big, 8);
      QCHECK(cudaMemcpyAsync(st, init, sizeof init, cudaMemcpyHostToDevice, ctx().s));
      const i64 nc = 2 * (f->nlinks / 2) * g.Vh;
      k_long_check<<<std::min<i64>(grid_for(nc, 256), (i64)ctx().red_blocks), 256, 0, ctx().s>>>(
          f->d, f->nlinks, g.Vh, st, st + 1, st + 2);
      QLAUNCH();
      unsigned long long h[3];
      QCHECK(cudaMemcpyAsync(h, st, sizeof h, cudaMemcpyDeviceToHost, ctx().s));
      sync();
      dfree(st);
      double defect, cmax, cmin;
      memcpy(&defect, &h[0], 8); memcpy(&cmax, &h[1], 8); memcpy(&cmin, &h[2], 8);
      // exact to well below the 2^-15 storage precision
      if (cmax > 0 && defect < 1e-7 && (cmax - cmin) <= 1e-7 * cmax) { recon = 1; c_long = cmax; }
      log0(QOP_VERB_MED, "sloppy links: long-link defect %g, |c| in [%g, %g] -> recon %d\n", defect, cmin, cmax, recon);
    }
    s->aq = dmalloc((size_t)2 * nblk * q16_block_bytes(f->nlinks, recon != 0));
    const i64 nt = 2 * nblk * f->nlinks * QB;
    k_links_q16b<<<grid_for(nt, 256), 256, 0, ctx().s>>>((unsigned char *)s->aq, f->d, f->nlinks, g.Vh, nblk, recon,
                                                          c_long);
    QLAUNCH();
    s->recon = recon;
    s->c_long = c_long;
    s->recon_mode = want_recon;
  }
  if (lkfmt == LK_F32 && !s->f32) s->f32 = fla_convert<float, double>(f);
  return s;
}

LinksSloppy links_parity(SloppyLinks *s, int lkfmt, int p) {
  const i64 Vh = ctx().g.Vh;
  const i64 o = (i64)p * s->nl * Vh;
  if (lkfmt == LK_F16)
    return LinksSloppy{(const uint4 *)s->a16 + o, (const uint4 *)s->b16 + o, (const __half2 *)s->c16 + o};
  if (lkfmt == LK_Q16) {
    const i64 nblk = (Vh + QB - 1) / QB;
    return LinksSloppy{(const unsigned char *)s->aq + (size_t)p * nblk * q16_block_bytes(s->nl, s->recon != 0),
                       nullptr, nullptr};
  }
  return LinksSloppy{s->f32->d + (i64)p * s->nl * 9 * Vh, nullptr, nullptr};
}

// int16 hop launch: variant 0 = plain loads, 4 slots batched;
// 1 / 2 = TMA bulk staging with 2- / 4-slot groups; 3 / 4 = plain loads
// with 2 / 8 slots batched; 5-10 = plain loads with the registers capped
// for B resident blocks per SM (5: 2 slots, B 10 = 48 registers; 6: 2, 12
// (spills); 7: 4, 8; 8: 2, 8; 9: 1, 10; 10: 2, 9); 11-16 = the same with a
// persistent grid of (SMs x B) blocks striding over the site blocks
// (11: 2, 10 (spills); 12: 2, 8; 13: 2, 7; 14: 4, 8; 15: 2, 6 = 80
// registers, the default; 16: 1, 8).  At 32^3x64 a hop takes 115.7 us with
// variant 15, 116-117 us with 12-14 and 16, 131 us with 5 and 149 us with 3
// (no register cap, ~150 registers): the persistent grid removes the
// partial last wave of blocks, the register cap matters less once it does.
// 17-19 = persistent with a per-thread cp.async ring 3 / 2 / 4 slots ahead
// (6 / 8 / 5 blocks per SM): 157-170 us, the 4-5 small asynchronous copies
// per slot and thread cost more issue slots than the latency they hide.
// 20-28 = persistent with packed FP32x2 arithmetic (q16_slot_pk): 2 slots
// and 6 / 7 / 8 blocks per SM, 4 slots and 6 / 7 / 5, 8 slots and 6, 4 and
// 8 slots with 4 blocks (128 registers; with the fused update the solve
// takes 1525 / 1536 ms against 1489 ms for 25 on one box).  At
// 32^3x64: 109.1-109.4 us with 25 (4 slots, 5 blocks, 96 registers; the
// default), 110.0 with 23, 111.2 with 20 / 21, 112-113 with 22, 24, 26,
// against 117.3 for the scalar variant 15 (a third fewer instructions per
// slot; the kernel was issue-bound at 62 % issue-active).
// 29-31 = 25 with an L2 bulk prefetch of the link stream 2 / 4 / 1 slot
// batches ahead: slower at 32^3x64 (hop / fused hop 118.1 / 123.4,
// 118.7 / 121.4 and 135.0 / 139.6 us against 113.0 / 119.2 us for 25, same
// box), the block's own loads already keep HBM as busy as the prefetches do.
// decomposed lattice: the hop of variant 25 (4 slots, 5 blocks per SM,
// persistent, packed) reading the halos of gh; KIND 1 or 3
static void launch_q16_dd(int kind, int nl, bool recon, float c_long, int grid, uint4 *out, const uint4 *src,
                          const unsigned char *lk, const uint4 *same, const Geom &g, const NbrGeom &ng, int par,
                          MixState *st, const uint4 *rres, int seq, const DdQ16Ghost &gh) {
  Context &c = ctx();
  const int gp = std::min(grid, (c.red_blocks / 8) * 5);
#define QDD_ARGS out, src, lk, same, g, ng, par, st, c.d_part, c.d_count, c_long, rres, seq, gh
#define QDD(K)                                                                                              \
  do {                                                                                                      \
    if (nl != 16) k_mix_hop_q16r<8, K, 4, false, 5, true, true, true><<<gp, QB, 0, c.s>>>(QDD_ARGS);        \
    else if (recon) k_mix_hop_q16r<16, K, 4, true, 5, true, true, true><<<gp, QB, 0, c.s>>>(QDD_ARGS);      \
    else k_mix_hop_q16r<16, K, 4, false, 5, true, true, true><<<gp, QB, 0, c.s>>>(QDD_ARGS);                \
  } while (0)
  if (kind == 1) QDD(1);
  else QDD(3);
#undef QDD
#undef QDD_ARGS
}

// KIND 3 hops (fused update) exist for the persistent packed variants 20-26
static void launch_q16_fused(int variant, int nl, bool recon, float c_long, int grid, uint4 *out, const uint4 *src,
                             const unsigned char *lk, const uint4 *same, const Geom &g, const NbrGeom &ng, int par,
                             MixState *st, const uint4 *rres, int seq, bool pdl = false) {
  Context &c = ctx();
#define Q16_ARGS3 out, src, lk, same, g, ng, par, st, c.d_part, c.d_count, c_long, rres, seq, DdQ16Ghost()
#define Q16RPK3(B, M)                                                                                          \
  do {                                                                                                         \
    const int gp = std::min(grid, (c.red_blocks / 8) * M);                                                     \
    if (nl != 16) launch_k(pdl, k_mix_hop_q16r<8, 3, B, false, M, true, true>, gp, QB, c.s, Q16_ARGS3);       \
    else if (recon) launch_k(pdl, k_mix_hop_q16r<16, 3, B, true, M, true, true>, gp, QB, c.s, Q16_ARGS3);     \
    else launch_k(pdl, k_mix_hop_q16r<16, 3, B, false, M, true, true>, gp, QB, c.s, Q16_ARGS3);               \
  } while (0)
#define Q16RPK3F(B, M, F)                                                                                           \
  do {                                                                                                              \
    const int gp = std::min(grid, (c.red_blocks / 8) * M);                                                          \
    if (nl != 16) launch_k(pdl, k_mix_hop_q16r<8, 3, B, false, M, true, true, false, F>, gp, QB, c.s, Q16_ARGS3);   \
    else if (recon) launch_k(pdl, k_mix_hop_q16r<16, 3, B, true, M, true, true, false, F>, gp, QB, c.s, Q16_ARGS3); \
    else launch_k(pdl, k_mix_hop_q16r<16, 3, B, false, M, true, true, false, F>, gp, QB, c.s, Q16_ARGS3);           \
  } while (0)
  switch (variant) {
    case 20: Q16RPK3(2, 6); break;
    case 21: Q16RPK3(2, 7); break;
    case 22: Q16RPK3(2, 8); break;
    case 23: Q16RPK3(4, 6); break;
    case 24: Q16RPK3(4, 7); break;
    case 26: Q16RPK3(8, 6); break;
    case 27: Q16RPK3(4, 4); break;
    case 28: Q16RPK3(8, 4); break;
    case 29: Q16RPK3F(4, 5, 2); break;
    case 30: Q16RPK3F(4, 5, 4); break;
    case 31: Q16RPK3F(4, 5, 1); break;
    default: Q16RPK3(4, 5); break;
  }
#undef Q16RPK3F
#undef Q16RPK3
#undef Q16_ARGS3
}

template <int KIND>
static void launch_q16(int variant, int nl, bool recon, float c_long, int grid, uint4 *out, const uint4 *src,
                       const unsigned char *lk, const uint4 *same, const Geom &g, const NbrGeom &ng, int par,
                       MixState *st, bool pdl = false) {
  Context &c = ctx();
#define Q16_ARGS out, src, lk, same, g, ng, par, st, c.d_part, c.d_count
#define Q16R(NLV, B)                                                                        \
  do {                                                                                      \
    if (recon) k_mix_hop_q16r<NLV, KIND, B, true><<<grid, QB, 0, c.s>>>(Q16_ARGS, c_long);  \
    else k_mix_hop_q16r<NLV, KIND, B, false><<<grid, QB, 0, c.s>>>(Q16_ARGS, c_long);       \
  } while (0)
#define Q16RM(B, M)                                                                                       \
  do {                                                                                                    \
    if (nl != 16) k_mix_hop_q16r<8, KIND, B, false, M><<<grid, QB, 0, c.s>>>(Q16_ARGS, c_long);          \
    else if (recon) k_mix_hop_q16r<16, KIND, B, true, M><<<grid, QB, 0, c.s>>>(Q16_ARGS, c_long);        \
    else k_mix_hop_q16r<16, KIND, B, false, M><<<grid, QB, 0, c.s>>>(Q16_ARGS, c_long);                  \
  } while (0)
#define Q16RP(B, M)                                                                                       \
  do {                                                                                                    \
    const int gp = std::min(grid, (c.red_blocks / 8) * M);                                                \
    if (nl != 16) k_mix_hop_q16r<8, KIND, B, false, M, true><<<gp, QB, 0, c.s>>>(Q16_ARGS, c_long);      \
    else if (recon) k_mix_hop_q16r<16, KIND, B, true, M, true><<<gp, QB, 0, c.s>>>(Q16_ARGS, c_long);    \
    else k_mix_hop_q16r<16, KIND, B, false, M, true><<<gp, QB, 0, c.s>>>(Q16_ARGS, c_long);              \
  } while (0)
#define Q16PK_TAIL c_long, (const uint4 *)nullptr, 0, DdQ16Ghost()
#define Q16RPK(B, M)                                                                                           \
  do {                                                                                                         \
    const int gp = std::min(grid, (c.red_blocks / 8) * M);                                                     \
    if (nl != 16) launch_k(pdl, k_mix_hop_q16r<8, KIND, B, false, M, true, true>, gp, QB, c.s, Q16_ARGS, Q16PK_TAIL);   \
    else if (recon) launch_k(pdl, k_mix_hop_q16r<16, KIND, B, true, M, true, true>, gp, QB, c.s, Q16_ARGS, Q16PK_TAIL); \
    else launch_k(pdl, k_mix_hop_q16r<16, KIND, B, false, M, true, true>, gp, QB, c.s, Q16_ARGS, Q16PK_TAIL);           \
  } while (0)
#define Q16RPKF(B, M, F)                                                                                      \
  do {                                                                                                         \
    const int gp = std::min(grid, (c.red_blocks / 8) * M);                                                     \
    if (nl != 16)                                                                                              \
      launch_k(pdl, k_mix_hop_q16r<8, KIND, B, false, M, true, true, false, F>, gp, QB, c.s, Q16_ARGS, Q16PK_TAIL);  \
    else if (recon)                                                                                            \
      launch_k(pdl, k_mix_hop_q16r<16, KIND, B, true, M, true, true, false, F>, gp, QB, c.s, Q16_ARGS, Q16PK_TAIL);  \
    else                                                                                                       \
      launch_k(pdl, k_mix_hop_q16r<16, KIND, B, false, M, true, true, false, F>, gp, QB, c.s, Q16_ARGS, Q16PK_TAIL); \
  } while (0)
#define Q16A(RR, M)                                                                                       \
  do {                                                                                                    \
    const int gp = std::min(grid, (c.red_blocks / 8) * M);                                                \
    if (nl != 16) k_mix_hop_q16a<8, KIND, false, RR, M><<<gp, QB, 0, c.s>>>(Q16_ARGS, c_long);            \
    else if (recon) k_mix_hop_q16a<16, KIND, true, RR, M><<<gp, QB, 0, c.s>>>(Q16_ARGS, c_long);          \
    else k_mix_hop_q16a<16, KIND, false, RR, M><<<gp, QB, 0, c.s>>>(Q16_ARGS, c_long);                    \
  } while (0)
  switch (variant) {
    case 5: Q16RM(2, 10); break;   // register cap for 10 resident blocks
    case 6: Q16RM(2, 12); break;
    case 7: Q16RM(4, 8); break;
    case 8: Q16RM(2, 8); break;
    case 9: Q16RM(1, 10); break;
    case 10: Q16RM(2, 9); break;
    case 11: Q16RP(2, 10); break;   // persistent grid of SMs x 10 blocks
    case 12: Q16RP(2, 8); break;
    case 13: Q16RP(2, 7); break;
    case 14: Q16RP(4, 8); break;
    case 15: Q16RP(2, 6); break;
    case 16: Q16RP(1, 8); break;
    case 17: Q16A(3, 6); break;    // cp.async ring of 3 slots ahead
    case 18: Q16A(2, 8); break;
    case 19: Q16A(4, 5); break;
    case 20: Q16RPK(2, 6); break;   // persistent, packed FP32x2 arithmetic
    case 21: Q16RPK(2, 7); break;
    case 22: Q16RPK(2, 8); break;
    case 23: Q16RPK(4, 6); break;
    case 24: Q16RPK(4, 7); break;
    case 25: Q16RPK(4, 5); break;
    case 26: Q16RPK(8, 6); break;
    case 27: Q16RPK(4, 4); break;
    case 28: Q16RPK(8, 4); break;
    case 29: Q16RPKF(4, 5, 2); break;   // 25 with an L2 prefetch two slot batches ahead
    case 30: Q16RPKF(4, 5, 4); break;   // ... one site block ahead
    case 31: Q16RPKF(4, 5, 1); break;   // ... one slot batch ahead
    case 1:
      if (nl == 16) k_mix_hop_q16<16, KIND, 2><<<grid, QB, 4 * QSLOT, c.s>>>(Q16_ARGS);
      else k_mix_hop_q16<8, KIND, 2><<<grid, QB, 4 * QSLOT, c.s>>>(Q16_ARGS);
      break;
    case 2:
      if (nl == 16) k_mix_hop_q16<16, KIND, 4><<<grid, QB, 8 * QSLOT, c.s>>>(Q16_ARGS);
      else k_mix_hop_q16<8, KIND, 4><<<grid, QB, 8 * QSLOT, c.s>>>(Q16_ARGS);
      break;
    case 3:
      if (nl == 16) Q16R(16, 2);
      else k_mix_hop_q16r<8, KIND, 2, false><<<grid, QB, 0, c.s>>>(Q16_ARGS, c_long);
      break;
    case 4:
      if (nl == 16) Q16R(16, 8);
      else k_mix_hop_q16r<8, KIND, 8, false><<<grid, QB, 0, c.s>>>(Q16_ARGS, c_long);
      break;
    default:
      if (nl == 16) Q16R(16, 4);
      else k_mix_hop_q16r<8, KIND, 4, false><<<grid, QB, 0, c.s>>>(Q16_ARGS, c_long);
      break;
  }
#undef Q16A
#undef Q16RPK
#undef Q16PK_TAIL
#undef Q16RP
#undef Q16RM
#undef Q16R
#undef Q16_ARGS
}

// ---------------------------------------------------------------- driver
// Shifted systems solved alongside the base one: sigma[0] = 0 is the base,
// stop[s] the absolute target on zeta_s^2 |r|^2, x[s] the FP64 solutions
// (x[0] is the base solution argument of run_mixed).
struct MsArgs {
  int ns;
  const double *sigma, *stop;
  c2<double> **x;
};

// autotuned int16 hop variant per (lattice extents, links per site, long-link
// reconstruction)
static std::map<std::array<int, 6>, int> g_hop_tuned;

template <class Sp, class Lk>
static void run_mixed(LinOp<double> &L, QOP_invert_arg_t *ia, QOP_resid_arg_t *ra, c2<double> *x,
                      const c2<double> *b, int eo, SloppyLinks *sl, int lkfmt, const MsArgs *ms = nullptr) {
  typedef typename Sp::elem E;
  Context &c = ctx();
  const Geom &g = c.g;
  const i64 Vh = g.Vh;
  const int p = eo, q = 1 - eo;
  const Range is = vrange(g, eo);
  const int ns = ms ? ms->ns : 1;
  const double b2 = Blas<double>::norm2(b, is);
  ra->final_rel = 0;
  ra->final_restart = 0;
  Blas<double>::zero(x, is);
  for (int s = 1; s < ns; s++) Blas<double>::zero(ms->x[s], is);
  if (b2 == 0.0) { ra->final_rsq = 0; ra->final_iter = 0; return; }
  need_finite(b2, "mixed solver: source norm");
  const double stop = ra->rsqmin * b2;
  const i64 nb = Sp::block(Vh);
  E *rs = nullptr, *ps = nullptr, *Aps = nullptr, *ts = nullptr;
  float2 *xs = nullptr;
  c2<double> *r = nullptr, *Ax = nullptr;
  MixState *dst = nullptr;
  MixState h{};
  MsShift *dsh = nullptr;
  MsVecs mv{};
  // frees every buffer of the solve (idempotent; on every exit, normal or
  // thrown, so that a failed allocation or a failed check leaks nothing)
  auto release = [&]() {
    dfree(rs); dfree(ps); dfree(Aps); dfree(ts); dfree(xs); dfree(r); dfree(Ax); dfree(dst);
    for (int s = 1; s < ns; s++) { dfree(mv.p[s]); dfree(mv.x[s]); mv.p[s] = nullptr; mv.x[s] = nullptr; }
    dfree(dsh);
    rs = ps = Aps = ts = nullptr; xs = nullptr; r = Ax = nullptr; dst = nullptr; dsh = nullptr;
  };
  try {
  rs = dalloc<E>(nb); ps = dalloc<E>(nb); Aps = dalloc<E>(nb); ts = dalloc<E>(nb);
  xs = dalloc<float2>(3 * Vh);
  dzero(xs, sizeof(float2) * 3 * Vh);
  r = dalloc<c2<double>>(vec_elems(g)); Ax = dalloc<c2<double>>(vec_elems(g));
  Blas<double>::copy(r, b, is);
  dst = dalloc<MixState>(1);
  if (ns > 1) {
    std::vector<MsShift> hs(ns);
    for (int s = 0; s < ns; s++) hs[s] = MsShift{ms->sigma[s], 1.0, 1.0, -1.0, ms->stop[s], 0.0, 1, 0};
    dsh = dalloc<MsShift>(ns);
    QCHECK(cudaMemcpyAsync(dsh, hs.data(), sizeof(MsShift) * ns, cudaMemcpyHostToDevice, c.s));
    for (int s = 1; s < ns; s++) {
      mv.p[s] = dalloc<E>(nb);
      mv.x[s] = dalloc<float2>(3 * Vh);
      dzero(mv.x[s], sizeof(float2) * 3 * Vh);
    }
  }
  const LinksSloppy lk_p = links_parity(sl, lkfmt, p), lk_q = links_parity(sl, lkfmt, q);
  const int gridh = grid_for(Vh, 128), gridv = grid_for(Vh, 256), gridq = (int)((Vh + QB - 1) / QB);
  NbrGeom ng;
  for (int d = 0; d < 4; d++) ng.L[d] = g.L[d];
  ng.str[3] = 1; ng.str[2] = g.L[3]; ng.str[1] = g.L[2] * g.L[3]; ng.str[0] = g.L[1] * g.L[2] * g.L[3];
  const int nl = sl->nl;
  // compulsory bytes: links once (reconstructed long links 28 B), input and
  // output sites once
  const double link_site = (std::is_same<Lk, LkQ16B>::value && sl->recon) ? (nl / 2) * (40.0 + 28.0)
                                                                           : (double)nl * Lk::link_bytes;
  const double hop_bytes = (double)Vh * (link_site + 2 * Sp::site_bytes);
  const bool recon = sl->recon != 0;
  const float c_long = (float)sl->c_long;
  char hname[32], hname3[40];
  snprintf(hname, sizeof hname, "hop_%s_link%s", Sp::name(), Lk::name());
  snprintf(hname3, sizeof hname3, "hop_%s_upd_link%s", Sp::name(), Lk::name());   // the fused-update hop

  auto refresh = [&](double r2) {   // sloppy r <- r, new residual reference
    k_to_sloppy<Sp><<<gridv, 256, 0, c.s>>>(rs, r + is.off, Vh);
    QLAUNCH();
    h.rsq = r2;
    h.maxr2 = r2;
  };
  h.stop = stop;
  h.mbar_tries = c.opt.mbar_tries;
  h.delta2 = c.opt.ru_delta * c.opt.ru_delta;
  h.m2 = L.mass * L.mass;
  h.max_iter = ia->max_iter;
  h.iter = 0;
  h.flag = MIX_RUN;
  refresh(b2);
  h.rsq_old = b2;
  k_copy_elems<E><<<grid_for(nb, 256), 256, 0, c.s>>>(ps, rs, nb);
  QLAUNCH();
  for (int s = 1; s < ns; s++) {
    k_copy_elems<E><<<grid_for(nb, 256), 256, 0, c.s>>>((E *)mv.p[s], rs, nb);
    QLAUNCH();
  }
  QCHECK(cudaMemcpyAsync(dst, &h, sizeof h, cudaMemcpyHostToDevice, c.s));
  int nru = 0, stalls = 0;
  double r2 = b2;
  const int chunk = c.opt.chunk;
  // fused update (option fuse_update): the second hop reduces what the
  // update needs and one kernel updates x, r and p
  constexpr bool q16v = std::is_same<Lk, LkQ16B>::value && std::is_same<Sp, SpQ16>::value;
  // int16 hop variant: the option, or (hop_kernel -1) the fastest of the
  // packed persistent variants 20-26 timed on this lattice's first solve
  int hk = c.opt.hop_kernel;
  if constexpr (std::is_same<Lk, LkQ16B>::value) {
    if (hk < 0) {
      const std::array<int, 6> key{g.L[0], g.L[1], g.L[2], g.L[3], nl, recon ? 1 : 0};
      auto it = g_hop_tuned.find(key);
      if (dd_active()) {
        hk = 25;   // the decomposed hop has the shape of variant 25
      } else if (it != g_hop_tuned.end()) {
        hk = it->second;
      } else {
        const unsigned char *lq = (const unsigned char *)lk_q.a;
        hk = tune_pick({20, 21, 22, 23, 24, 25, 26}, [&](int v) {   // t = D p: recomputed by the first iteration
          launch_q16<1>(v, nl, recon, c_long, gridq, ts, ps, lq, nullptr, g, ng, q, dst);
          QLAUNCH();
        });
        g_hop_tuned[key] = hk;
        log0(QOP_VERB_LOW, "autotune: int16 hop variant %d on %dx%dx%dx%d\n", hk, g.L[0], g.L[1], g.L[2], g.L[3]);
      }
    }
  }
  const bool fuse = q16v && c.opt.fuse_update && hk >= 20;
  // the three kernels of the fused iteration as programmatic dependents
  const bool pdl = fuse && c.opt.pdl;
  int seq = 0;
  // a decomposed lattice: halos before each hop, the reductions summed over
  // the processes before the scalars (the fused int16 iteration only)
  const bool ddq = dd_active();
  if (ddq && !fuse) {
    release();
    fail(QOP_FAIL, "mixed solver on a decomposed lattice: needs int16 storage, one mass, fuse_update and a "
                   "packed hop variant (20-26)");
  }
  while (true) {
    const int it0 = h.iter;
    int prof0 = -1;
    std::vector<int> recs;
    for (int k = 0; k < chunk; k++) {
      if constexpr (q16v) {
        if (ddq) {
          const unsigned char *lq = (const unsigned char *)lk_q.a, *lp = (const unsigned char *)lk_p.a;
          {
            ProfScope ps1(hname, hop_bytes);
            const DdQ16Ghost g1 = dd_halo_q16(nl, lp, recon, c_long, ps, p);
            launch_q16_dd(1, nl, recon, c_long, gridq, ts, ps, lq, nullptr, g, ng, q, dst, nullptr, 0, g1);
            recs.push_back(ps1.idx);
          }
          dd_allreduce(&dst->dp2, 1);
          {
            ProfScope ps2(hname3, hop_bytes + (double)Vh * Sp::site_bytes * 2);
            const DdQ16Ghost g2 = dd_halo_q16(nl, lq, recon, c_long, ts, q);
            launch_q16_dd(3, nl, recon, c_long, gridq, Aps, ts, lp, ps, g, ng, p, dst, rs, ++seq, g2);
            recs.push_back(ps2.idx);
          }
          dd_allreduce(dst->red3, 3);
          k_mix_scalars3<<<1, 1, 0, c.s>>>(dst, seq);
          k_mix_update_p<Sp><<<gridv, 256, 0, c.s>>>(xs, rs, ps, Aps, Vh, dst, seq);
          QLAUNCHN(4);
          continue;
        }
      }
      {
        ProfScope ps1(hname, hop_bytes);
        if constexpr (std::is_same<Lk, LkQ16B>::value) {
          const unsigned char *lq = (const unsigned char *)lk_q.a;
          launch_q16<1>(hk, nl, recon, c_long, gridq, ts, ps, lq, nullptr, g, ng, q, dst, pdl);
        } else {
          if (nl == 16) k_mix_hop<Sp, Lk, 16, 1><<<gridh, 128, 0, c.s>>>(ts, ps, lk_q, nullptr, g, q, dst, c.d_part, c.d_count);
          else k_mix_hop<Sp, Lk, 8, 1><<<gridh, 128, 0, c.s>>>(ts, ps, lk_q, nullptr, g, q, dst, c.d_part, c.d_count);
        }
        recs.push_back(ps1.idx);
      }
      {
        ProfScope ps2(fuse ? hname3 : hname, hop_bytes + (double)Vh * Sp::site_bytes * (fuse ? 2 : 1));
        if constexpr (q16v) {
          const unsigned char *lp = (const unsigned char *)lk_p.a;
          if (fuse) launch_q16_fused(hk, nl, recon, c_long, gridq, Aps, ts, lp, ps, g, ng, p, dst, rs, ++seq, pdl);
          else launch_q16<2>(hk, nl, recon, c_long, gridq, Aps, ts, lp, ps, g, ng, p, dst);
        } else if constexpr (std::is_same<Lk, LkQ16B>::value) {
          const unsigned char *lp = (const unsigned char *)lk_p.a;
          launch_q16<2>(hk, nl, recon, c_long, gridq, Aps, ts, lp, ps, g, ng, p, dst);
        } else {
          if (nl == 16) k_mix_hop<Sp, Lk, 16, 2><<<gridh, 128, 0, c.s>>>(Aps, ts, lk_p, ps, g, p, dst, c.d_part, c.d_count);
          else k_mix_hop<Sp, Lk, 8, 2><<<gridh, 128, 0, c.s>>>(Aps, ts, lk_p, ps, g, p, dst, c.d_part, c.d_count);
        }
        recs.push_back(ps2.idx);
      }
      if (ns > 1 && fuse) {
        {
          // compulsory bytes with every shift active: base x (FP32) rw, r rw,
          // p rw, Ap read; x_s rw and p_s rw per shift
          ProfScope pm("ms_update", (double)Vh * (48.0 + 5 * Sp::site_bytes + (ns - 1) * (48.0 + 2 * Sp::site_bytes)));
          launch_k(pdl, k_ms_update_fused<Sp>, gridv, 256, c.s, xs, rs, ps, (const E *)Aps, Vh, dst, seq, c.d_part,
                   c.d_count, dsh, ns, mv);
        }
        QLAUNCHN(3);
      } else if (ns > 1) {
        {
          // compulsory bytes with every shift active: base x (FP32) rw, r rw,
          // p and Ap read, x_s rw and p_s read per shift; then p rw, r read,
          // p_s rw per shift
          ProfScope pm("ms_update", (double)Vh * (4 * Sp::site_bytes + 48.0 + (ns - 1) * (48.0 + Sp::site_bytes) +
                                                  3 * Sp::site_bytes + (ns - 1) * 2 * Sp::site_bytes));
          k_ms_update<Sp><<<gridv, 256, 0, c.s>>>(xs, rs, ps, Aps, Vh, dst, c.d_part, c.d_count, dsh, ns, mv);
          k_ms_p<Sp><<<gridv, 256, 0, c.s>>>(ps, rs, Vh, dst, dsh, ns, mv);
        }
        QLAUNCHN(4);
      } else if (fuse) {
        launch_k(pdl, k_mix_update_p<Sp>, gridv, 256, c.s, xs, rs, ps, (const E *)Aps, Vh, (const MixState *)dst, seq);
        QLAUNCHN(3);
      } else {
        k_mix_update<Sp><<<gridv, 256, 0, c.s>>>(xs, rs, ps, Aps, Vh, dst, c.d_part, c.d_count);
        k_mix_p<Sp><<<gridv, 256, 0, c.s>>>(ps, rs, Vh, dst);
        QLAUNCHN(4);
      }
    }
    (void)prof0;
    QCHECK(cudaMemcpyAsync(&h, dst, sizeof h, cudaMemcpyDeviceToHost, c.s));
    sync();
    // drop timing records of launches that found the flag set (no work)
    int ran = h.iter - it0;                       // completed iterations
    int hops_ran = 2 * ran + (h.flag == MIX_BREAK ? 2 : 0);
    for (size_t k = hops_ran; k < recs.size(); k++) prof_discard(recs[k]);
    if (h.flag == MIX_RUN) continue;
    if (h.flag == MIX_ERROR) {
      release();
      fail(QOP_FAIL, "mixed solver: a bulk copy into shared memory did not complete in time");
    }
    stalls = ran == 0 ? stalls + 1 : 0;           // repeated breakdown without progress
    // reliable update: fold the sloppy solution into FP64, true residual
    k_fold_x<<<grid_for(3 * Vh, 256), 256, 0, c.s>>>(x + is.off, xs, 3 * Vh);
    QLAUNCH();
    for (int s = 1; s < ns; s++) {
      k_fold_x<<<grid_for(3 * Vh, 256), 256, 0, c.s>>>(ms->x[s] + is.off, mv.x[s], 3 * Vh);
      QLAUNCH();
    }
    L.d2(Ax, x);
    Blas<double>::axpby(r, 1.0, b, -1.0, Ax, is);
    r2 = Blas<double>::norm2(r, is);
    need_finite(r2, "mixed solver: true residual norm");
    nru++;
    log0(QOP_VERB_MED, "MIXCG[%d]: iter %d sloppy rsq %g true rsq %g (stop %g)\n", lkfmt, h.iter, h.rsq, r2, stop);
    if (r2 <= stop || h.iter + nru >= h.max_iter || stalls > 2) break;
    const bool broke = (h.flag == MIX_BREAK);
    const double rsq_prev = broke ? 0.0 : h.rsq_old;
    if (ns > 1 && (broke || !(rsq_prev > 0))) break;   // shifted recurrences cannot restart
    refresh(r2);
    if (broke || !(rsq_prev > 0)) {
      // restart the recursion from the true residual
      k_copy_elems<E><<<grid_for(nb, 256), 256, 0, c.s>>>(ps, rs, nb);
      QLAUNCH();
    } else {
      h.beta = r2 / rsq_prev;
      h.flag = MIX_RUN;
      QCHECK(cudaMemcpyAsync(dst, &h, sizeof h, cudaMemcpyHostToDevice, c.s));
      if (ns > 1) k_ms_p<Sp><<<gridv, 256, 0, c.s>>>(ps, rs, Vh, dst, dsh, ns, mv);
      else k_mix_p<Sp><<<gridv, 256, 0, c.s>>>(ps, rs, Vh, dst);
      QLAUNCH();
    }
    h.flag = MIX_RUN;
    QCHECK(cudaMemcpyAsync(dst, &h, sizeof h, cudaMemcpyHostToDevice, c.s));
  }
  ra->final_rsq = r2 / b2;
  ra->final_iter = h.iter + nru;
  release();
  sync();
  } catch (...) {
    release();
    throw;
  }
}

static void run_sloppy(LinOp<double> &L, QOP_invert_arg_t *ia, QOP_resid_arg_t *ra, c2<double> *x,
                       const c2<double> *b, int eo, int prec, const MsArgs *ms) {
  if (prec == 32) {
    run_mixed<SpF32, LkF32>(L, ia, ra, x, b, eo, sloppy_get(L.f, LK_F32), LK_F32, ms);
    return;
  }
  // 16-bit storage: 0 = int16 fixed point (default), 1 = IEEE FP16,
  // 2 = FP16 links with int16 vectors
  switch (ctx().opt.half_format) {
    case 1: run_mixed<SpF16, LkF16>(L, ia, ra, x, b, eo, sloppy_get(L.f, LK_F16), LK_F16, ms); break;
    case 2: run_mixed<SpQ16, LkF16>(L, ia, ra, x, b, eo, sloppy_get(L.f, LK_F16), LK_F16, ms); break;
    default: run_mixed<SpQ16, LkQ16B>(L, ia, ra, x, b, eo, sloppy_get(L.f, LK_Q16), LK_Q16, ms); break;
  }
}

bool mixed_cgms(LinOp<double> &L, QOP_invert_arg_t *ia, QOP_resid_arg_t **ra, const double *shifts, int ns,
                c2<double> **out, const c2<double> *in, int eo, int prec) {
  if (ns != 1 || shifts[0] != 0.0) return false;   // multi-shift: reference CGMS in FP64
  if (prec != 16 && prec != 32) return false;
  run_sloppy(L, ia, ra[0], out[0], in, eo, prec, nullptr);
  return true;
}

// Several masses and/or sources on one parity with sloppy storage.
// With int16 storage every solve runs in one batched reliable-update CG
// (batch.cu): the systems share each hop's link stream, so heavier masses
// and further sources ride along with the slowest system at little extra
// cost, and each keeps the convergence of its own single-mass solve.
// Otherwise (or with the option multi_shift = 1) the solves that share a
// source and start from zero first run as one reduced-precision multi-shift
// CG (reliable updates on the lightest mass; every heavier mass stops when
// its implied residual zeta^2 |r|^2 reaches its target), and every solve is
// then refined from that vector to its FP64 target (batched with int16
// storage, else through the reference driver one solve at a time).  The
// shifted solutions of the first phase are only as accurate as the sloppy
// recurrences let them be: each reliable update of the base residual moves
// the shifted residuals by zeta_s times the base's accumulated rounding
// drift.  Solves with a Fermilab relative-norm target go through the
// reference driver.
void solve_multi_mixed(QOP_info_t *info, FlaT<double> *f, QOP_invert_arg_t *ia, QOP_resid_arg_t **ra,
                       const double *masses, c2<double> **out, c2<double> **in, int nsolve) {
  const Geom &g = ctx().g;
  const Options &o = ctx().opt;
  const int eo = ia->evenodd, prec = o.sloppy_prec;
  const Range is = vrange(g, eo);
  const double t0 = wtime();
  const double nflop = 0.5 * (20 * 3 + 2 * 8 * 3 * 3 * f->nlinks), nflopm = 0.5 * 10 * 3;
  const int max_iter = ia->max_iter;
  const bool batched = prec == 16 && o.half_format == 0;
  double flop = 0;
  int it1 = 0;
  std::vector<char> seen(nsolve, 0);
  for (int i = 0; i < nsolve && (!batched || o.multi_shift); i++) {
    if (seen[i]) continue;
    std::vector<int> grp;
    for (int j = i; j < nsolve; j++)
      if (!seen[j] && in[j] == in[i]) { grp.push_back(j); seen[j] = 1; }
    std::vector<double> m2;
    bool ok = true;
    for (int j : grp) {
      m2.push_back(masses[j] * masses[j]);
      if (ra[j]->relmin > 0) ok = false;
    }
    std::sort(m2.begin(), m2.end());
    m2.erase(std::unique(m2.begin(), m2.end()), m2.end());
    const int ns = (int)m2.size();
    if (!ok || ns < 2 || ns > MS_MAX) continue;
    for (int j : grp)
      if (Blas<double>::norm2(out[j], is) != 0.0) ok = false;
    const double b2 = Blas<double>::norm2(in[i], is);
    if (!ok || b2 == 0.0) continue;
    std::vector<double> sigma(ns), stop(ns, -1.0);
    for (int s = 0; s < ns; s++) sigma[s] = m2[s] - m2[0];
    // The shifted systems are refined afterwards, and their phase-1
    // residuals cannot fall below the sloppy operator's drift, (eps kappa_s)^2
    // relative with eps ~ 2^-15 for int16 storage (>= 1e-9 for kappa_s >= 1):
    // they stop at ms_stop (by default 1e-10 with int16 storage), which
    // spares the update of shifts that can no longer improve.  The lightest
    // mass keeps its own target.
    const double ms_stop = o.ms_stop >= 0 ? o.ms_stop : (batched ? 1e-10 : 0.0);
    for (int j : grp) {
      const int s = (int)(std::lower_bound(m2.begin(), m2.end(), masses[j] * masses[j]) - m2.begin());
      const double t = (s > 0 ? std::max(ra[j]->rsqmin, ms_stop) : ra[j]->rsqmin) * b2;
      stop[s] = stop[s] < 0 ? t : std::min(stop[s], t);
    }
    ScopedVecs own;   // the phase's vectors
    std::vector<c2<double> *> xv(ns);
    for (int s = 0; s < ns; s++) xv[s] = own.add();
    c2<double> *tmp = own.add();
    LinOp<double> L{f, std::sqrt(m2[0]), eo, tmp};
    QOP_invert_arg_t ia1 = *ia;
    QOP_resid_arg_t ra1 = QOP_RESID_ARG_DEFAULT;
    ra1.rsqmin = stop[0] / b2;
    const MsArgs msa{ns, sigma.data(), stop.data(), xv.data()};
    run_sloppy(L, &ia1, &ra1, xv[0], in[i], eo, prec, &msa);
    it1 += ra1.final_iter;
    flop += (nflop + nflopm * (ns - 1)) * ra1.final_iter * (double)g.V;
    if (ctx().verbosity >= QOP_VERB_MED) {
      c2<double> *ax = own.add();
      for (int s = 0; s < ns; s++) {
        LinOp<double> Ls{f, std::sqrt(m2[s]), eo, tmp};
        Ls.d2(ax, xv[s]);
        Blas<double>::axpby(ax, 1.0, in[i], -1.0, ax, is);
        log0(QOP_VERB_MED, "SOLVE(mixed multi-mass): mass %g true rsq %g target %g\n", std::sqrt(m2[s]),
             Blas<double>::norm2(ax, is) / b2, stop[s] / b2);
      }
    }
    for (int j : grp) {
      const int s = (int)(std::lower_bound(m2.begin(), m2.end(), masses[j] * masses[j]) - m2.begin());
      Blas<double>::copy(out[j], xv[s], is);
    }
  }
  int it2 = 0, nres = 0;
  std::vector<int> bat;
  for (int i = 0; i < nsolve; i++) {
    if (batched && ra[i]->relmin <= 0) { bat.push_back(i); continue; }
    QOP_info_t inf{};
    QOP_invert_arg_t ia2 = *ia;
    ia2.max_iter = std::max(1, max_iter - it1);
    solve_multi<double>(&inf, f, &ia2, &ra[i], &masses[i], &out[i], &in[i], 1);
    it2 = std::max(it2, ra[i]->final_iter);
    nres = std::max(nres, ra[i]->final_restart);
    ra[i]->final_iter += it1;
    flop += inf.final_flop;
  }
  for (size_t c0 = 0; c0 < bat.size(); c0 += BATCH_MAX) {
    const int n = (int)std::min<size_t>(BATCH_MAX, bat.size() - c0);
    std::vector<double> m(n), rq(n), frs(n);
    std::vector<c2<double> *> xs(n), bs(n);
    std::vector<int> its(n);
    for (int k = 0; k < n; k++) {
      const int i = bat[c0 + k];
      m[k] = masses[i]; rq[k] = ra[i]->rsqmin; xs[k] = out[i]; bs[k] = in[i];
    }
    run_batch(f, eo, n, m.data(), xs.data(), bs.data(), rq.data(), std::max(1, max_iter - it1), its.data(),
              frs.data());
    for (int k = 0; k < n; k++) {
      const int i = bat[c0 + k];
      Blas<double>::scale(out[i], masses[i], out[i], is);   // m A^{-1} in
      ra[i]->final_rsq = frs[k];
      ra[i]->final_rel = 0;
      ra[i]->final_iter = it1 + its[k];
      ra[i]->final_restart = 0;
      it2 = std::max(it2, its[k]);
      flop += nflop * its[k] * (double)g.V;
    }
  }
  log0(QOP_VERB_LOW, "SOLVE(mixed multi-mass): multi-shift its %d, refinement its %d\n", it1, it2);
  sync();
  if (info) {
    info->final_sec = wtime() - t0;
    info->final_flop = flop;
    info->status = QOP_SUCCESS;
  }
}

}  // namespace qopb

// ---------------------------------------------------------------- test entry point
namespace qopb {
// int16 parity block -> FP64 [3][Vh] parity block (the stored values)
__global__ void k_q16_to_f64(double2 *d, const uint4 *s, i64 Vh) {
  const i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (i >= Vh) return;
  float2 v[3];
  SpQ16::load(s, (int)i, Vh, v);
#pragma unroll
  for (int c = 0; c < 3; c++) d[c * Vh + i] = make_double2(v[c].x, v[c].y);
}
}  // namespace qopb

// The int16 normal-equation operator of the mixed solver, applied once with
// the solver's own kernels: p = int16(in) on parity eo, t = D_oe p (the
// first hop, stored as int16 on the other parity) and Ap = m^2 p - D_eo t
// (the second hop: kind 2, or kind 3 = the fused-update hop that also
// reduces <p, Ap> and |Ap|^2).  t and Ap are decoded into t_out / ap_out.
// sums[0..3] = |t|^2, |p|^2, <p, Ap>, |Ap|^2 as the kernels reduced them
// (the last two only for kind 3).  Restates QOP_asqtad_ddagd_norm2
// (lib/asqtad_dslash_p.c:1121-1138) in the solver's storage; it exists so
// that the sloppy operator can be compared site by site with FP64.
extern "C" int QOPB_D3_sloppy_ddagd(QOP_info_t *info, QOP_D3_FermionLinksAsqtad *asqtad, double mass,
                                    QOP_D3_ColorVector *t_out, QOP_D3_ColorVector *ap_out, QOP_D3_ColorVector *in,
                                    QOP_evenodd_t eo, int variant, int kind2, double *sums) {
  using namespace qopb;
  uint4 *p16 = nullptr, *t16 = nullptr, *a16 = nullptr;
  MixState *dst = nullptr;
  try {
    require_init("QOPB_D3_sloppy_ddagd");
    dd_refuse("QOPB_D3_sloppy_ddagd");
    handle_check(asqtad, "FermionLinksAsqtad");
    handle_check(t_out, "ColorVector");
    handle_check(ap_out, "ColorVector");
    handle_check(in, "ColorVector");
    if (eo != QOP_EVEN && eo != QOP_ODD) fail(QOP_FAIL, "QOPB_D3_sloppy_ddagd: eo must be EVEN or ODD");
    if (variant < 0 || variant > 28) fail(QOP_FAIL, "QOPB_D3_sloppy_ddagd: hop variant %d (0..28)", variant);
    if (kind2 != 2 && kind2 != 3) fail(QOP_FAIL, "QOPB_D3_sloppy_ddagd: second hop kind %d (2 or 3)", kind2);
    if (kind2 == 3 && variant < 20) fail(QOP_FAIL, "QOPB_D3_sloppy_ddagd: kind 3 needs a packed variant (20..28)");
    FlaT<double> *f = reinterpret_cast<FlaT<double> *>(asqtad);
    VecT<double> *to = reinterpret_cast<VecT<double> *>(t_out), *ao = reinterpret_cast<VecT<double> *>(ap_out);
    VecT<double> *vi = reinterpret_cast<VecT<double> *>(in);
    Context &c = ctx();
    const Geom &g = c.g;
    const i64 Vh = g.Vh;
    const int p = eo, q = 1 - eo;
    SloppyLinks *sl = sloppy_get(f, LK_Q16);
    const LinksSloppy lk_p = links_parity(sl, LK_Q16, p), lk_q = links_parity(sl, LK_Q16, q);
    p16 = dalloc<uint4>(Vh);
    t16 = dalloc<uint4>(Vh);
    a16 = dalloc<uint4>(Vh);
    dst = dalloc<MixState>(1);
    MixState h{};
    h.flag = MIX_RUN;
    h.m2 = mass * mass;
    h.rsq = h.rsq_old = h.maxr2 = 1.0;
    h.max_iter = 1 << 30;
    QCHECK(cudaMemcpyAsync(dst, &h, sizeof h, cudaMemcpyHostToDevice, c.s));
    const int gridv = grid_for(Vh, 256), gridq = (int)((Vh + QB - 1) / QB);
    NbrGeom ng;
    for (int d = 0; d < 4; d++) ng.L[d] = g.L[d];
    ng.str[3] = 1; ng.str[2] = g.L[3]; ng.str[1] = g.L[2] * g.L[3]; ng.str[0] = g.L[1] * g.L[2] * g.L[3];
    k_to_sloppy<SpQ16><<<gridv, 256, 0, c.s>>>(p16, vi->d + par_off(g, p), Vh);
    QLAUNCH();
    const bool recon = sl->recon != 0;
    const float c_long = (float)sl->c_long;
    launch_q16<1>(variant, sl->nl, recon, c_long, gridq, t16, p16, (const unsigned char *)lk_q.a, nullptr, g, ng, q,
                  dst);
    QLAUNCH();
    if (kind2 == 3)
      launch_q16_fused(variant, sl->nl, recon, c_long, gridq, a16, t16, (const unsigned char *)lk_p.a, p16, g, ng, p,
                       dst, p16, 1);
    else
      launch_q16<2>(variant, sl->nl, recon, c_long, gridq, a16, t16, (const unsigned char *)lk_p.a, p16, g, ng, p,
                    dst);
    QLAUNCH();
    k_q16_to_f64<<<gridv, 256, 0, c.s>>>(to->d + par_off(g, q), t16, Vh);
    k_q16_to_f64<<<gridv, 256, 0, c.s>>>(ao->d + par_off(g, p), a16, Vh);
    QLAUNCHN(2);
    QCHECK(cudaMemcpyAsync(&h, dst, sizeof h, cudaMemcpyDeviceToHost, c.s));
    sync();
    if (sums) {
      sums[0] = h.dp2;
      sums[1] = kind2 == 3 ? h.red3[0] : h.red;
      sums[2] = kind2 == 3 ? h.red3[1] : 0.0;
      sums[3] = kind2 == 3 ? h.red3[2] : 0.0;
    }
    dfree(p16); dfree(t16); dfree(a16); dfree(dst);
    if (info) info->status = QOP_SUCCESS;
    return 0;
  } catch (Fail &e) {
    dfree(p16); dfree(t16); dfree(a16); dfree(dst);
    fprintf(stderr, "QOPB_D3_sloppy_ddagd: %s\n", e.msg.c_str());
    if (info) info->status = e.status;
    return -1;
  }
}
