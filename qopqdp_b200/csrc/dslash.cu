// dslash.cu -- asqtad/HISQ Dslash in the handle's precision (FP64 / FP32).
// Reference: lib/asqtad_dslash_p.c:1048-1092 (eo dispatch), :1246-1279
// (style-1 hop: dest = sum_k dbllinks[k](x) src(x + shift_k)), :1019-1023
// (mass term), :1106-1138 (ddagd, ddagd_norm2), :1166-1191 (dslash_dir).
#include "reduce.cuh"
#include "dslash.cuh"
#include "dd.cuh"
#include "prof.cuh"

namespace qopb {

enum HopMode {
  HOP_SET = 0,      // out = hop
  HOP_MASS = 1,     // out = mass*same + hop
  HOP_MASS_ALIAS = 2,  // out = mass*hop + hop  (reference result when out == in)
  HOP_M2_MINUS = 3  // out = mass*same - hop   (ddagd epilogue, mass = m^2)
};

// neighbour (mu, d) of site x for a hop: the input vector, or on a
// decomposed lattice the up halo when the hop leaves the block upwards.
// Returns false when the term is a down-halo product, already added to a.
template <typename T, bool DD>
__device__ __forceinline__ bool hop_input(const Geom &g, const int x[4], int mu, int d, const c2<T> *src,
                                          const DdGhost<T> &gh, c2<T> &v0, c2<T> &v1, c2<T> &v2, c2<T> *a) {
  const i64 Vh = g.Vh;
  if (DD && (gh.mask >> mu & 1) && (unsigned)(x[mu] + d) >= (unsigned)g.L[mu]) {
    const int y = x[mu] + d, fh = gh.fh[mu], fi = dd_face_index(g, x, mu);
    const int sl = dd_halo_slab(g.L[mu], y, d);
    if (y < 0) {   // slab 0: the fat product at y = -1; slab -y: the long product
      const c2<T> *G = gh.dn[mu] + (i64)(sl * 3) * fh + fi;
      a[0] = cadd<T>(a[0], G[0]); a[1] = cadd<T>(a[1], G[fh]); a[2] = cadd<T>(a[2], G[2 * fh]);
      return false;
    }
    const c2<T> *G = gh.up[mu] + (i64)(sl * 3) * fh + fi;
    v0 = G[0]; v1 = G[fh]; v2 = G[2 * fh];
    return true;
  }
  const int j = nbr_index(g, x, mu, d);
  v0 = src[j]; v1 = src[Vh + j]; v2 = src[2 * Vh + j];
  return true;
}

// RED: 0 none, 1 = sum |out|^2, 2 = sum |same|^2; DD: read halos (dd.cuh)
template <typename T, int NL, int MODE, int RED, bool DD = false>
__global__ void __launch_bounds__(128)
k_hop(c2<T> *__restrict__ out, const c2<T> *__restrict__ src, const c2<T> *__restrict__ lk,
      const c2<T> *__restrict__ same, T mass, Geom g, int p,
      double *part, unsigned *count, double *res, DdGhost<T> gh = DdGhost<T>()) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const i64 Vh = g.Vh;
  double racc[1] = {0.0};
  if (i < Vh) {
    int x[4];
    site_coords(g, i, p, x);
    c2<T> a[3] = {mk<T>(0, 0), mk<T>(0, 0), mk<T>(0, 0)};
#pragma unroll
    for (int k = 0; k < NL; k++) {
      c2<T> v0, v1, v2;
      if (!hop_input<T, DD>(g, x, slot_mu<NL>(k), slot_disp<NL>(k), src, gh, v0, v1, v2, a)) continue;
      const c2<T> *U = lk + (i64)k * 9 * Vh + i;
      cfma<T>(a[0], U[0], v0); cfma<T>(a[0], U[Vh], v1); cfma<T>(a[0], U[2 * Vh], v2);
      cfma<T>(a[1], U[3 * Vh], v0); cfma<T>(a[1], U[4 * Vh], v1); cfma<T>(a[1], U[5 * Vh], v2);
      cfma<T>(a[2], U[6 * Vh], v0); cfma<T>(a[2], U[7 * Vh], v1); cfma<T>(a[2], U[8 * Vh], v2);
    }
    const c2<T> a0 = a[0], a1 = a[1], a2 = a[2];
    c2<T> r0, r1, r2;
    if (MODE == HOP_SET) { r0 = a0; r1 = a1; r2 = a2; }
    else if (MODE == HOP_MASS_ALIAS) {
      r0 = mk<T>(mass * a0.x + a0.x, mass * a0.y + a0.y);
      r1 = mk<T>(mass * a1.x + a1.x, mass * a1.y + a1.y);
      r2 = mk<T>(mass * a2.x + a2.x, mass * a2.y + a2.y);
    } else {
      const c2<T> s0 = same[i], s1 = same[Vh + i], s2 = same[2 * Vh + i];
      if (MODE == HOP_MASS) {
        r0 = mk<T>(mass * s0.x + a0.x, mass * s0.y + a0.y);
        r1 = mk<T>(mass * s1.x + a1.x, mass * s1.y + a1.y);
        r2 = mk<T>(mass * s2.x + a2.x, mass * s2.y + a2.y);
      } else {
        r0 = mk<T>(mass * s0.x - a0.x, mass * s0.y - a0.y);
        r1 = mk<T>(mass * s1.x - a1.x, mass * s1.y - a1.y);
        r2 = mk<T>(mass * s2.x - a2.x, mass * s2.y - a2.y);
      }
      if (RED == 2)
        racc[0] = (double)s0.x * s0.x + (double)s0.y * s0.y + (double)s1.x * s1.x + (double)s1.y * s1.y +
                  (double)s2.x * s2.x + (double)s2.y * s2.y;
    }
    out[i] = r0; out[Vh + i] = r1; out[2 * Vh + i] = r2;
    if (RED == 1)
      racc[0] = (double)r0.x * r0.x + (double)r0.y * r0.y + (double)r1.x * r1.x + (double)r1.y * r1.y +
                (double)r2.x * r2.x + (double)r2.y * r2.y;
  }
  if (RED) grid_sum<1>(racc, part, count, res);
}

// one direction, weighted, accumulating (style-1 dslash_dir)
template <typename T, int NL, bool DD = false>
__global__ void k_hop_dir(c2<T> *__restrict__ out, const c2<T> *__restrict__ src, const c2<T> *__restrict__ lk,
                          int k0, int nk, T w0, T w1, Geom g, int p, DdGhost<T> gh = DdGhost<T>()) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const i64 Vh = g.Vh;
  if (i >= Vh) return;
  int x[4];
  site_coords(g, i, p, x);
  c2<T> a[3] = {out[i], out[Vh + i], out[2 * Vh + i]};
  for (int kk = 0; kk < nk; kk++) {
    const int k = k0 + kk;
    const T w = kk == 0 ? w0 : w1;
    c2<T> u0, u1, u2;
    c2<T> h[3] = {mk<T>(0, 0), mk<T>(0, 0), mk<T>(0, 0)};
    if (!hop_input<T, DD>(g, x, slot_mu<NL>(k), slot_disp<NL>(k), src, gh, u0, u1, u2, h)) {
      for (int r = 0; r < 3; r++) a[r] = cadd<T>(a[r], cscale<T>(w, h[r]));   // w (-U^+ psi)
      continue;
    }
    c2<T> v[3] = {cscale<T>(w, u0), cscale<T>(w, u1), cscale<T>(w, u2)};
    const c2<T> *U = lk + (i64)k * 9 * Vh + i;
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) cfma<T>(a[r], U[(3 * r + c) * Vh], v[c]);
  }
  out[i] = a[0]; out[Vh + i] = a[1]; out[2 * Vh + i] = a[2];
}

template <typename T, int MODE>
struct FMass {   // out = mass*in (+ out) on a parity range
  c2<T> *out; const c2<T> *in; T mass;
  __device__ void operator()(i64 i) const {
    c2<T> v = in[i];
    if (MODE == 0) out[i] = mk<T>(mass * v.x, mass * v.y);
    else { c2<T> o = out[i]; out[i] = mk<T>(mass * v.x + o.x, mass * v.y + o.y); }
  }
};

constexpr int HOP_BLOCK = 128;

template <typename T, int MODE, int RED>
static void launch_hop(FlaT<T> *f, c2<T> *out, const c2<T> *in, const c2<T> *same, double mass, int p,
                       double *res) {
  Context &c = ctx();
  const Geom &g = c.g;
  const i64 lk_par = (i64)f->nlinks * 9 * g.Vh;
  c2<T> *o = out + par_off(g, p);
  const c2<T> *src = in + par_off(g, 1 - p);
  const c2<T> *lk = f->d + p * lk_par;
  const c2<T> *sm = same ? same + par_off(g, p) : nullptr;
  int grid = grid_for(g.Vh, HOP_BLOCK);
  // compulsory bytes: every link once, the input and output vectors once,
  // plus the same-parity input of the fused mass / m^2 epilogues
  const double bytes = (double)g.Vh * sizeof(T) * 2 *
                       (f->nlinks * 9 + 3 + 3 + ((MODE == HOP_MASS || MODE == HOP_M2_MINUS) ? 3 : 0));
  if (dd_active()) {
    const DdGhost<T> gh = dd_halo<T>(f, src, 1 - p);
    ProfScope ps(sizeof(T) == 8 ? "hop_f64_dd" : "hop_f32_dd", bytes);
    if (f->nlinks == 16)
      k_hop<T, 16, MODE, RED, true><<<grid, HOP_BLOCK, 0, c.s>>>(o, src, lk, sm, (T)mass, g, p, c.d_part, c.d_count,
                                                                 res, gh);
    else
      k_hop<T, 8, MODE, RED, true><<<grid, HOP_BLOCK, 0, c.s>>>(o, src, lk, sm, (T)mass, g, p, c.d_part, c.d_count,
                                                                res, gh);
    QLAUNCH();
    return;
  }
  ProfScope ps(sizeof(T) == 8 ? "hop_f64" : "hop_f32", bytes);
  if (f->nlinks == 16)
    k_hop<T, 16, MODE, RED><<<grid, HOP_BLOCK, 0, c.s>>>(o, src, lk, sm, (T)mass, g, p, c.d_part, c.d_count, res);
  else
    k_hop<T, 8, MODE, RED><<<grid, HOP_BLOCK, 0, c.s>>>(o, src, lk, sm, (T)mass, g, p, c.d_part, c.d_count, res);
  QLAUNCH();
}

template <typename T>
void Dslash<T>::hop(FlaT<T> *f, c2<T> *out, const c2<T> *in, int p) {
  launch_hop<T, HOP_SET, 0>(f, out, in, nullptr, 0.0, p, nullptr);
}

// hop on subset eo (the reference's asqtad_hop macro); when mass_sum is set
// the reference's following mass_term(out, in, mass, out) is fused in
template <typename T>
static void hop_sub(FlaT<T> *f, c2<T> *out, const c2<T> *in, int eo, bool mass_sum, double mass) {
  const Geom &g = ctx().g;
  const bool alias = (out == in);
  if (eo == QOP_EVENODD) {
    const c2<T> *src = in;
    c2<T> *tmp = nullptr;
    if (alias) {   // the even half is overwritten before the odd half is read
      tmp = dalloc<c2<T>>(vec_elems(g));
      Blas<T>::copy(tmp, in, vrange(g, QOP_EVENODD));
      src = tmp;
    }
    for (int p = 0; p < 2; p++) {
      if (!mass_sum) launch_hop<T, HOP_SET, 0>(f, out, src, nullptr, 0.0, p, nullptr);
      else if (alias) launch_hop<T, HOP_MASS_ALIAS, 0>(f, out, src, nullptr, mass, p, nullptr);
      else launch_hop<T, HOP_MASS, 0>(f, out, src, in, mass, p, nullptr);
    }
    if (tmp) dfree(tmp);
    return;
  }
  const int p = eo;
  if (!mass_sum) launch_hop<T, HOP_SET, 0>(f, out, in, nullptr, 0.0, p, nullptr);
  else if (alias) launch_hop<T, HOP_MASS_ALIAS, 0>(f, out, in, nullptr, mass, p, nullptr);
  else launch_hop<T, HOP_MASS, 0>(f, out, in, in, mass, p, nullptr);
}

template <typename T>
static void mass_term(c2<T> *out, const c2<T> *in, double mass, bool sum, int eo) {
  Range r = vrange(ctx().g, eo);
  if (!sum) run_map(FMass<T, 0>{out + r.off, in + r.off, (T)mass}, r.n);
  else run_map(FMass<T, 1>{out + r.off, in + r.off, (T)mass}, r.n);
}

template <typename T>
void Dslash<T>::apply(FlaT<T> *f, double mass, c2<T> *out, const c2<T> *in, int eo_out, int eo_in) {
  if (eo_in == eo_out) {
    if (eo_out == QOP_EVENODD) hop_sub<T>(f, out, in, QOP_EVENODD, true, mass);
    else mass_term<T>(out, in, mass, false, eo_out);
    return;
  }
  if (eo_out == QOP_EVEN || eo_out == QOP_EVENODD) {
    if (eo_in == QOP_ODD) hop_sub<T>(f, out, in, QOP_EVEN, false, 0);
    else if (eo_in == QOP_EVEN) mass_term<T>(out, in, mass, false, QOP_EVEN);
    else hop_sub<T>(f, out, in, QOP_EVEN, true, mass);
  }
  if (eo_out == QOP_ODD || eo_out == QOP_EVENODD) {
    if (eo_in == QOP_EVEN) hop_sub<T>(f, out, in, QOP_ODD, false, 0);
    else if (eo_in == QOP_ODD) mass_term<T>(out, in, mass, false, QOP_ODD);
    else hop_sub<T>(f, out, in, QOP_ODD, true, mass);
  }
}

template <typename T>
void Dslash<T>::dslash_dir(FlaT<T> *f, int dir, int fb, double wtfat, double wtlong, c2<T> *out,
                           const c2<T> *in, int eo_out) {
  Context &c = ctx();
  const Geom &g = c.g;
  int k0, nk;
  if (f->nlinks == 16) { k0 = fb > 0 ? 4 * dir : 4 * dir + 2; nk = 2; }
  else { k0 = fb > 0 ? 2 * dir : 2 * dir + 1; nk = 1; }
  const c2<T> *src = in;
  c2<T> *tmp = nullptr;
  if (out == in && eo_out == QOP_EVENODD) {
    tmp = dalloc<c2<T>>(vec_elems(g));
    Blas<T>::copy(tmp, in, vrange(g, QOP_EVENODD));
    src = tmp;
  }
  const i64 lk_par = (i64)f->nlinks * 9 * g.Vh;
  for (int p = 0; p < 2; p++) {
    if (eo_out != QOP_EVENODD && eo_out != p) continue;
    int grid = grid_for(g.Vh, HOP_BLOCK);
    if (dd_active()) {
      const DdGhost<T> gh = dd_halo<T>(f, src + par_off(g, 1 - p), 1 - p);
      if (f->nlinks == 16)
        k_hop_dir<T, 16, true><<<grid, HOP_BLOCK, 0, c.s>>>(out + par_off(g, p), src + par_off(g, 1 - p),
                                                            f->d + p * lk_par, k0, nk, (T)wtfat, (T)wtlong, g, p, gh);
      else
        k_hop_dir<T, 8, true><<<grid, HOP_BLOCK, 0, c.s>>>(out + par_off(g, p), src + par_off(g, 1 - p),
                                                           f->d + p * lk_par, k0, nk, (T)wtfat, (T)wtlong, g, p, gh);
      QLAUNCH();
      continue;
    }
    if (f->nlinks == 16)
      k_hop_dir<T, 16><<<grid, HOP_BLOCK, 0, c.s>>>(out + par_off(g, p), src + par_off(g, 1 - p), f->d + p * lk_par,
                                                     k0, nk, (T)wtfat, (T)wtlong, g, p);
    else
      k_hop_dir<T, 8><<<grid, HOP_BLOCK, 0, c.s>>>(out + par_off(g, p), src + par_off(g, 1 - p), f->d + p * lk_par,
                                                    k0, nk, (T)wtfat, (T)wtlong, g, p);
    QLAUNCH();
  }
  if (tmp) dfree(tmp);
}

template <typename T>
double Dslash<T>::ddagd(FlaT<T> *f, double mass, c2<T> *out, const c2<T> *in, int eo, c2<T> *tmp, bool want_norm) {
  Context &c = ctx();
  const int p = eo, q = 1 - eo;
  const T m2 = (T)mass * (T)mass;
  if (!want_norm) {
    launch_hop<T, HOP_SET, 0>(f, tmp, in, nullptr, 0.0, q, nullptr);
    launch_hop<T, HOP_M2_MINUS, 0>(f, out, tmp, in, (double)m2, p, nullptr);
    return 0.0;
  }
  launch_hop<T, HOP_SET, 1>(f, tmp, in, nullptr, 0.0, q, c.d_res);
  launch_hop<T, HOP_M2_MINUS, 2>(f, out, tmp, in, (double)m2, p, c.d_res + 1);
  dd_allreduce(c.d_res, 2);
  QCHECK(cudaMemcpyAsync(c.h_res, c.d_res, 2 * sizeof(double), cudaMemcpyDeviceToHost, c.s));
  QCHECK(cudaStreamSynchronize(c.s));
  // the reference returns |D in|^2 + m^2 |in|^2 in the working precision
  return (double)((T)c.h_res[0] + m2 * (T)c.h_res[1]);
}

template <typename T>
void Dslash<T>::ddagd_norm2_ws(FlaT<T> *f, double mass, c2<T> *out, const c2<T> *in, int eo, c2<T> *tmp_block,
                               double *part, unsigned *count, double *res) {
  Context &c = ctx();
  const Geom &g = c.g;
  const int p = eo, q = 1 - eo;
  const T m2 = (T)mass * (T)mass;
  const i64 lk_par = (i64)f->nlinks * 9 * g.Vh;
  const int grid = grid_for(g.Vh, HOP_BLOCK);
  // t = D_qp in (sum |t|^2 -> res[0]); out_p = m^2 in_p - D_pq t (sum |in_p|^2 -> res[1])
  if (f->nlinks == 16) {
    k_hop<T, 16, HOP_SET, 1><<<grid, HOP_BLOCK, 0, c.s>>>(tmp_block, in + par_off(g, p), f->d + q * lk_par, nullptr,
                                                          (T)0, g, q, part, count, res);
    k_hop<T, 16, HOP_M2_MINUS, 2><<<grid, HOP_BLOCK, 0, c.s>>>(out + par_off(g, p), tmp_block, f->d + p * lk_par,
                                                               in + par_off(g, p), m2, g, p, part, count, res + 1);
  } else {
    k_hop<T, 8, HOP_SET, 1><<<grid, HOP_BLOCK, 0, c.s>>>(tmp_block, in + par_off(g, p), f->d + q * lk_par, nullptr,
                                                         (T)0, g, q, part, count, res);
    k_hop<T, 8, HOP_M2_MINUS, 2><<<grid, HOP_BLOCK, 0, c.s>>>(out + par_off(g, p), tmp_block, f->d + p * lk_par,
                                                              in + par_off(g, p), m2, g, p, part, count, res + 1);
  }
  QLAUNCHN(2);
}

template struct Dslash<float>;
template struct Dslash<double>;

}  // namespace qopb
