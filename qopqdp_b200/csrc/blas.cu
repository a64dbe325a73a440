// blas.cu -- level-1 operations on checkerboarded vectors (the QDP_V_* and
// QDP_r_eq_* calls of lib/invert_cg_p.c and lib/asqtad_invert_p.c).
// A parity block is contiguous ([parity][colour][site]), so every subset
// operation is a flat unit-stride loop over complex elements.
#include "reduce.cuh"

namespace qopb {

namespace {

template <typename T> struct FZero { c2<T> *v; __device__ void operator()(i64 i) const { v[i] = mk<T>(0, 0); } };
template <typename T> struct FCopy {
  c2<T> *d; const c2<T> *s;
  __device__ void operator()(i64 i) const { d[i] = s[i]; }
};
template <typename T> struct FScale {
  c2<T> *d; const c2<T> *s; double a;
  __device__ void operator()(i64 i) const { c2<T> v = s[i]; d[i] = mk<T>((T)(a * v.x), (T)(a * v.y)); }
};
template <typename T> struct FCScale {
  c2<T> *d; const c2<T> *s; double ar, ai;
  __device__ void operator()(i64 i) const {
    c2<T> v = s[i];
    d[i] = mk<T>((T)(ar * v.x - ai * v.y), (T)(ar * v.y + ai * v.x));
  }
};
template <typename T> struct FAxpy {
  c2<T> *y; const c2<T> *x; T a;
  __device__ void operator()(i64 i) const { c2<T> u = y[i], v = x[i]; y[i] = mk<T>(u.x + a * v.x, u.y + a * v.y); }
};
template <typename T> struct FCAxpy {
  c2<T> *y; const c2<T> *x; T ar, ai;
  __device__ void operator()(i64 i) const {
    c2<T> u = y[i], v = x[i];
    y[i] = mk<T>(u.x + ar * v.x - ai * v.y, u.y + ar * v.y + ai * v.x);
  }
};
template <typename T> struct FXpay {
  c2<T> *y; const c2<T> *x; T a;
  __device__ void operator()(i64 i) const { c2<T> u = y[i], v = x[i]; y[i] = mk<T>(v.x + a * u.x, v.y + a * u.y); }
};
template <typename T> struct FAxpby {
  c2<T> *z; const c2<T> *x; const c2<T> *y; T a, b;
  __device__ void operator()(i64 i) const {
    c2<T> u = x[i], v = y[i];
    z[i] = mk<T>(a * u.x + b * v.x, a * u.y + b * v.y);
  }
};
template <typename T> struct FCAxpby {
  c2<T> *z; const c2<T> *x; const c2<T> *y; T ar, ai;
  __device__ void operator()(i64 i) const {
    c2<T> u = x[i], v = y[i];
    z[i] = mk<T>(ar * u.x - ai * u.y + v.x, ar * u.y + ai * u.x + v.y);
  }
};
template <typename T> struct RNorm {
  const c2<T> *v;
  __device__ void operator()(i64 i, double *acc) const {
    c2<T> u = v[i];
    acc[0] += (double)u.x * u.x + (double)u.y * u.y;
  }
};
template <typename T> struct RDot {
  const c2<T> *a; const c2<T> *b;
  __device__ void operator()(i64 i, double *acc) const {
    c2<T> u = a[i], v = b[i];
    acc[0] += (double)u.x * v.x + (double)u.y * v.y;
    acc[1] += (double)u.x * v.y - (double)u.y * v.x;
  }
};
template <typename T> struct RCgUpd {
  c2<T> *x; c2<T> *r; const c2<T> *p; const c2<T> *Ap; T a;
  __device__ void operator()(i64 i, double *acc) const {
    c2<T> xv = x[i], rv = r[i], pv = p[i], av = Ap[i];
    xv.x += a * pv.x; xv.y += a * pv.y;
    rv.x -= a * av.x; rv.y -= a * av.y;
    x[i] = xv; r[i] = rv;
    acc[0] += (double)rv.x * rv.x + (double)rv.y * rv.y;
  }
};
template <typename T> struct RRel {
  const c2<T> *r; const c2<T> *x; i64 Vh; int p0;
  __device__ void operator()(i64 s, double *acc) const {
    int p = p0 + (int)(s / Vh);
    i64 i = s % Vh;
    i64 base = (i64)p * 3 * Vh + i;
    double xn = 0, rn = 0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      c2<T> xv = x[base + c * Vh], rv = r[base + c * Vh];
      xn += (double)xv.x * xv.x + (double)xv.y * xv.y;
      rn += (double)rv.x * rv.x + (double)rv.y * rv.y;
    }
    acc[0] += (xn == 0.0) ? 1.0 : rn / xn;
  }
};
template <typename TD, typename TS> struct FConv {
  c2<TD> *d; const c2<TS> *s;
  __device__ void operator()(i64 i) const { c2<TS> v = s[i]; d[i] = mk<TD>((TD)v.x, (TD)v.y); }
};

}  // namespace

template <typename T> void Blas<T>::zero(c2<T> *v, Range r) { run_map(FZero<T>{v + r.off}, r.n); }
template <typename T> void Blas<T>::copy(c2<T> *d, const c2<T> *s, Range r) {
  if (d == s) return;
  run_map(FCopy<T>{d + r.off, s + r.off}, r.n);
}
template <typename T> void Blas<T>::scale(c2<T> *d, double a, const c2<T> *s, Range r) {
  run_map(FScale<T>{d + r.off, s + r.off, a}, r.n);
}
template <typename T> void Blas<T>::cscale(c2<T> *d, dcx a, const c2<T> *s, Range r) {
  run_map(FCScale<T>{d + r.off, s + r.off, a.re, a.im}, r.n);
}
template <typename T> void Blas<T>::axpy(c2<T> *y, double a, const c2<T> *x, Range r) {
  run_map(FAxpy<T>{y + r.off, x + r.off, (T)a}, r.n);
}
template <typename T> void Blas<T>::caxpy(c2<T> *y, dcx a, const c2<T> *x, Range r) {
  run_map(FCAxpy<T>{y + r.off, x + r.off, (T)a.re, (T)a.im}, r.n);
}
template <typename T> void Blas<T>::xpay(c2<T> *y, const c2<T> *x, double a, Range r) {
  run_map(FXpay<T>{y + r.off, x + r.off, (T)a}, r.n);
}
template <typename T> void Blas<T>::axpby(c2<T> *z, double a, const c2<T> *x, double b, const c2<T> *y, Range r) {
  run_map(FAxpby<T>{z + r.off, x + r.off, y + r.off, (T)a, (T)b}, r.n);
}
template <typename T> void Blas<T>::caxpby(c2<T> *z, dcx a, const c2<T> *x, const c2<T> *y, Range r) {
  run_map(FCAxpby<T>{z + r.off, x + r.off, y + r.off, (T)a.re, (T)a.im}, r.n);
}
template <typename T> double Blas<T>::norm2(const c2<T> *v, Range r) {
  double s;
  run_reduce<1>(RNorm<T>{v + r.off}, r.n, &s);
  return s;
}
template <typename T> dcx Blas<T>::cdot(const c2<T> *a, const c2<T> *b, Range r) {
  double s[2];
  run_reduce<2>(RDot<T>{a + r.off, b + r.off}, r.n, s);
  return {s[0], s[1]};
}
template <typename T> double Blas<T>::redot(const c2<T> *a, const c2<T> *b, Range r) { return cdot(a, b, r).re; }
template <typename T>
double Blas<T>::cg_update(c2<T> *x, c2<T> *r, double a, const c2<T> *p, const c2<T> *Ap, Range q) {
  double s;
  run_reduce<1>(RCgUpd<T>{x + q.off, r + q.off, p + q.off, Ap + q.off, (T)a}, q.n, &s);
  return s;
}
template <typename T> double Blas<T>::relnorm_sum(const c2<T> *r, const c2<T> *x, int eo) {
  const Geom &g = ctx().g;
  double s;
  int p0 = eo == QOP_ODD ? 1 : 0;
  i64 n = eo == QOP_EVENODD ? 2 * g.Vh : g.Vh;
  run_reduce<1>(RRel<T>{r, x, g.Vh, p0}, n, &s);
  return s;
}

template <typename TD, typename TS> void convert(c2<TD> *d, const c2<TS> *s, Range r) {
  run_map(FConv<TD, TS>{d + r.off, s + r.off}, r.n);
}

template struct Blas<float>;
template struct Blas<double>;
template void convert<float, double>(c2<float> *, const c2<double> *, Range);
template void convert<double, float>(c2<double> *, const c2<float> *, Range);
template void convert<double, double>(c2<double> *, const c2<double> *, Range);
template void convert<float, float>(c2<float> *, const c2<float> *, Range);

}  // namespace qopb
