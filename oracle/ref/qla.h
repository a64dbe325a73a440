/* qla.h -- the QLA site types and site macros that the reference's asqtad
   path uses, for building it against qdp_shim (test infrastructure).
   Written from the call sites in QOPQDP (lib/asqtad_dslash_p.c,
   lib/asqtad_invert_p.c, lib/invert_cg_p.c): complex numbers are structs
   with .real / .imag, colour vectors hold Nc complex elements, colour
   matrices Nc x Nc row-major (`e[i][j]`, as lib/hisq_reunit_utilities_p.c
   and examples/test_reunit_utils.c access them).  Only Nc = 3 is computed
   with; the other colour types exist so that the reference's headers
   parse. */
#ifndef QLA_SHIM_H
#define QLA_SHIM_H
#include <math.h>

typedef float QLA_F_Real;
typedef double QLA_D_Real;
typedef struct { float real, imag; } QLA_F_Complex;
typedef struct { double real, imag; } QLA_D_Complex;
typedef int QLA_Int;

#define QLA_SHIM_COLOR_TYPES(P, NC, NCN)                                                          \
  typedef struct { QLA_##P##_Complex c[NC]; } QLA_##P##NCN##_ColorVector;                       \
  typedef struct { QLA_##P##_Complex e[NC][NC]; } QLA_##P##NCN##_ColorMatrix;                   \
  typedef struct { QLA_##P##_Complex d[4][NC]; } QLA_##P##NCN##_DiracFermion;                   \
  typedef struct { QLA_##P##_Complex h[2][NC]; } QLA_##P##NCN##_HalfFermion;                    \
  typedef struct { QLA_##P##_Complex p[4][NC][4][NC]; } QLA_##P##NCN##_DiracPropagator;

QLA_SHIM_COLOR_TYPES(F, 1, 1)
QLA_SHIM_COLOR_TYPES(D, 1, 1)
QLA_SHIM_COLOR_TYPES(F, 2, 2)
QLA_SHIM_COLOR_TYPES(D, 2, 2)
QLA_SHIM_COLOR_TYPES(F, 3, 3)
QLA_SHIM_COLOR_TYPES(D, 3, 3)
/* Nc = N types: declared with 3 colours so that prototypes parse */
QLA_SHIM_COLOR_TYPES(F, 3, N)
QLA_SHIM_COLOR_TYPES(D, 3, N)
#define QLA_FN_ColorVector(nc, x) QLA_FN_ColorVector x
#define QLA_FN_ColorMatrix(nc, x) QLA_FN_ColorMatrix x
#define QLA_FN_DiracFermion(nc, x) QLA_FN_DiracFermion x
#define QLA_DN_ColorVector(nc, x) QLA_DN_ColorVector x
#define QLA_DN_ColorMatrix(nc, x) QLA_DN_ColorMatrix x
#define QLA_DN_DiracFermion(nc, x) QLA_DN_DiracFermion x

/* precision-generic names (QLA_Precision / QLA_Colors set by the stub) */
#if defined(QLA_Precision) && QLA_Precision == 'F'
typedef QLA_F_Real QLA_Real;
typedef QLA_F_Complex QLA_Complex;
#define QLA_SHIM_PC(x) QLA_F3_##x
#else
typedef QLA_D_Real QLA_Real;
typedef QLA_D_Complex QLA_Complex;
#define QLA_SHIM_PC(x) QLA_D3_##x
#endif
typedef QLA_SHIM_PC(ColorVector) QLA_ColorVector;
typedef QLA_SHIM_PC(ColorMatrix) QLA_ColorMatrix;
typedef QLA_SHIM_PC(DiracFermion) QLA_DiracFermion;

typedef QLA_F3_ColorVector QLA_F_ColorVector;
typedef QLA_F3_ColorMatrix QLA_F_ColorMatrix;
typedef QLA_F3_DiracFermion QLA_F_DiracFermion;
typedef QLA_D3_ColorVector QLA_D_ColorVector;
typedef QLA_D3_ColorMatrix QLA_D_ColorMatrix;
typedef QLA_D3_DiracFermion QLA_D_DiracFermion;

/* complex macros: arguments are complex values (lvalues where assigned) */
#define QLA_real(c) ((c).real)
#define QLA_imag(c) ((c).imag)
#define QLA_c_eq_c(r, a) do { (r).real = (a).real; (r).imag = (a).imag; } while (0)
#define QLA_c_eqm_c(r, a) do { (r).real = -(a).real; (r).imag = -(a).imag; } while (0)
#define QLA_c_eq_r(r, x) do { (r).real = (x); (r).imag = 0; } while (0)
#define QLA_c_eq_r_plus_ir(c, x, y) do { (c).real = (x); (c).imag = (y); } while (0)
#define QLA_c_eq_r_times_c(r, x, a) do { (r).real = (x) * (a).real; (r).imag = (x) * (a).imag; } while (0)
#define QLA_c_peq_r_times_c(r, x, a) do { (r).real += (x) * (a).real; (r).imag += (x) * (a).imag; } while (0)
#define QLA_c_eq_c_div_r(r, a, x) do { (r).real = (a).real / (x); (r).imag = (a).imag / (x); } while (0)
#define QLA_norm2_c(a) ((a).real * (a).real + (a).imag * (a).imag)
#define QLA_c_eq_c_div_c(r, a, b)                                            \
  do {                                                                       \
    double _n = QLA_norm2_c(b);                                              \
    double _re = ((a).real * (b).real + (a).imag * (b).imag) / _n;           \
    double _im = ((a).imag * (b).real - (a).real * (b).imag) / _n;           \
    (r).real = _re; (r).imag = _im;                                          \
  } while (0)
#define QLA_c_eq_r_div_c(r, x, b)                                            \
  do {                                                                       \
    double _n = QLA_norm2_c(b);                                              \
    double _re = (x) * (b).real / _n, _im = -(x) * (b).imag / _n;            \
    (r).real = _re; (r).imag = _im;                                          \
  } while (0)

/* element access */
#define QLA_elem_V(v, i) ((v).c[i])
#define QLA_elem_M(m, i, j) ((m).e[i][j])

/* matrix macros: arguments are pointers */
#define QLA_M_eq_M(r, a) (*(r) = *(a))
#define QLA_M_eqm_M(r, a)                                                    \
  do {                                                                       \
    for (int _i = 0; _i < 3; _i++)                                           \
      for (int _j = 0; _j < 3; _j++) {                                       \
        (r)->e[_i][_j].real = -(a)->e[_i][_j].real;                          \
        (r)->e[_i][_j].imag = -(a)->e[_i][_j].imag;                          \
      }                                                                      \
  } while (0)
#define QLA_M_eq_c_times_M(r, c, a)                                          \
  do {                                                                       \
    for (int _i = 0; _i < 3; _i++)                                           \
      for (int _j = 0; _j < 3; _j++) {                                       \
        double _re = (c)->real * (a)->e[_i][_j].real - (c)->imag * (a)->e[_i][_j].imag; \
        double _im = (c)->real * (a)->e[_i][_j].imag + (c)->imag * (a)->e[_i][_j].real; \
        (r)->e[_i][_j].real = _re; (r)->e[_i][_j].imag = _im;                \
      }                                                                      \
  } while (0)
#define QLA_c_eq_c_times_c(r, a, b)                                          \
  do {                                                                       \
    double _re = (a).real * (b).real - (a).imag * (b).imag;                  \
    double _im = (a).real * (b).imag + (a).imag * (b).real;                  \
    (r).real = _re; (r).imag = _im;                                          \
  } while (0)
#define QLA_c_peq_c(r, a) do { (r).real += (a).real; (r).imag += (a).imag; } while (0)
#define QLA_c_peq_r(r, x) do { (r).real += (x); } while (0)
#define QLA_c_eq_c_plus_c(r, a, b)                                           \
  do {                                                                       \
    double _re = (a).real + (b).real, _im = (a).imag + (b).imag;             \
    (r).real = _re; (r).imag = _im;                                          \
  } while (0)
#define QLA_c_eq_c_minus_c(r, a, b)                                          \
  do {                                                                       \
    double _re = (a).real - (b).real, _im = (a).imag - (b).imag;             \
    (r).real = _re; (r).imag = _im;                                          \
  } while (0)
#define QLA_FD_C_eq_C(r, a) do { (r)->real = (a)->real; (r)->imag = (a)->imag; } while (0)
#define QLA_M_eq_zero(r)                                                     \
  do {                                                                       \
    for (int _i = 0; _i < 3; _i++)                                           \
      for (int _j = 0; _j < 3; _j++) (r)->e[_i][_j].real = (r)->e[_i][_j].imag = 0; \
  } while (0)
#define QLA_M_eq_Ma(r, a)                                                    \
  do {                                                                       \
    for (int _i = 0; _i < 3; _i++)                                           \
      for (int _j = 0; _j < 3; _j++) {                                       \
        (r)->e[_i][_j].real = (a)->e[_j][_i].real;                           \
        (r)->e[_i][_j].imag = -(a)->e[_j][_i].imag;                          \
      }                                                                      \
  } while (0)
#define QLA_M_eq_r_times_M(r, x, a)                                          \
  do {                                                                       \
    for (int _i = 0; _i < 3; _i++)                                           \
      for (int _j = 0; _j < 3; _j++) {                                       \
        (r)->e[_i][_j].real = *(x) * (a)->e[_i][_j].real;                    \
        (r)->e[_i][_j].imag = *(x) * (a)->e[_i][_j].imag;                    \
      }                                                                      \
  } while (0)
#define QLA_M_eq_r_times_M_plus_M(r, x, a, b)                                \
  do {                                                                       \
    for (int _i = 0; _i < 3; _i++)                                           \
      for (int _j = 0; _j < 3; _j++) {                                       \
        (r)->e[_i][_j].real = *(x) * (a)->e[_i][_j].real + (b)->e[_i][_j].real; \
        (r)->e[_i][_j].imag = *(x) * (a)->e[_i][_j].imag + (b)->e[_i][_j].imag; \
      }                                                                      \
  } while (0)
#define QLA_R_eq_re_trace_M(r, a) (*(r) = (a)->e[0][0].real + (a)->e[1][1].real + (a)->e[2][2].real)
/* r = op(a) op(b) into a temporary first (r may alias a or b); ta / tb: adjoint */
#define QLA_SHIM_MM(r, a, ta, b, tb)                                         \
  do {                                                                       \
    double _tr[3][3], _ti[3][3];                                             \
    for (int _i = 0; _i < 3; _i++)                                           \
      for (int _j = 0; _j < 3; _j++) {                                       \
        double _sr = 0, _si = 0;                                             \
        for (int _k = 0; _k < 3; _k++) {                                     \
          double _ar = (ta) ? (a)->e[_k][_i].real : (a)->e[_i][_k].real;     \
          double _ai = (ta) ? -(a)->e[_k][_i].imag : (a)->e[_i][_k].imag;    \
          double _br = (tb) ? (b)->e[_j][_k].real : (b)->e[_k][_j].real;     \
          double _bi = (tb) ? -(b)->e[_j][_k].imag : (b)->e[_k][_j].imag;    \
          _sr += _ar * _br - _ai * _bi;                                      \
          _si += _ar * _bi + _ai * _br;                                      \
        }                                                                    \
        _tr[_i][_j] = _sr; _ti[_i][_j] = _si;                                \
      }                                                                      \
    for (int _i = 0; _i < 3; _i++)                                           \
      for (int _j = 0; _j < 3; _j++) {                                       \
        (r)->e[_i][_j].real = _tr[_i][_j]; (r)->e[_i][_j].imag = _ti[_i][_j]; \
      }                                                                      \
  } while (0)
#define QLA_M_eq_M_times_M(r, a, b) QLA_SHIM_MM(r, a, 0, b, 0)
#define QLA_M_eq_M_times_Ma(r, a, b) QLA_SHIM_MM(r, a, 0, b, 1)
#define QLA_M_eq_Ma_times_M(r, a, b) QLA_SHIM_MM(r, a, 1, b, 0)
#define QLA_D_M_eq_M_times_M QLA_M_eq_M_times_M
#define QLA_D_M_eq_Ma_times_M QLA_M_eq_Ma_times_M
#define QLA_SHIM_CONV_M(r, a)                                                \
  do {                                                                       \
    for (int _i = 0; _i < 3; _i++)                                           \
      for (int _j = 0; _j < 3; _j++) {                                       \
        (r)->e[_i][_j].real = (a)->e[_i][_j].real;                           \
        (r)->e[_i][_j].imag = (a)->e[_i][_j].imag;                           \
      }                                                                      \
  } while (0)
#define QLA_DF_M_eq_M QLA_SHIM_CONV_M
#define QLA_FD_M_eq_M QLA_SHIM_CONV_M
/* the inverse square root of a positive Hermitian matrix is reached only by
   the reference's projection for Nc != 3 (lib/hisq_reunit2_p.c); Nc = 3 uses
   the analytic U(3) projection of lib/hisq_reunit_utilities_p.c */
#include <stdio.h>
#include <stdlib.h>
#define QLA_D_M_eq_invsqrtPH_M(r, a)                                         \
  do {                                                                       \
    fprintf(stderr, "qla shim: M_eq_invsqrtPH_M is not provided\n");       \
    abort();                                                                 \
  } while (0)
#define QLA_R_eq_norm2_V(r, a)                                               \
  do {                                                                       \
    double _s = 0;                                                           \
    for (int _i = 0; _i < 3; _i++) _s += QLA_norm2_c((a)->c[_i]);            \
    *(r) = _s;                                                               \
  } while (0)

#endif
