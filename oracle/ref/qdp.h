/* qdp.h -- the part of the QDP/C interface that the reference's asqtad
   path calls (fields, subsets, shifts, BLAS-1, reductions), implemented for
   one process on the CPU by qdp_shim.c / qdp_shim_p.c.  Test
   infrastructure: it lets the reference's own lib/asqtad_dslash_p.c,
   lib/asqtad_invert_p.c, lib/invert_cg_p.c, lib/invert_utilities_p.c,
   lib/asqtad_invert.c and lib/common.c be compiled, unmodified, into
   oracle/_ref/libqopref.so.  The names, argument order and meaning follow
   the reference's call sites (e.g. lib/asqtad_dslash_p.c:1218-1279 for the
   shifts, lib/invert_cg_p.c for the BLAS-1 and reductions).

   Site order: a field holds V sites in the QOP raw order (even sites first,
   lexicographic with x[0] slowest; lib/layout_user.c:237-258), so
   QDP_even / QDP_odd are the two halves and raw arrays are fields.
   Reductions accumulate in double for both precisions. */
#ifndef QDP_SHIM_H
#define QDP_SHIM_H
#include <stdlib.h>
#if defined(QDP_Precision) && !defined(QLA_Precision)
#define QLA_Precision QDP_Precision   /* QDP sets the precision of the generic QLA names */
#endif
#include "qla.h"
#include "qmp.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct QDP_Lattice_s QDP_Lattice;
typedef struct QDP_Layout_s QDP_Layout;
typedef struct QDP_RandomState_s QDP_RandomState;
struct QDP_Subset_s { int start, len; };
typedef struct QDP_Subset_s *QDP_Subset;
struct QDP_Shift_s { int disp[4]; int *fwd, *bck; };   /* neighbour index tables */
typedef struct QDP_Shift_s *QDP_Shift;
typedef enum { QDP_forward = 0, QDP_backward = 1 } QDP_ShiftDir;

extern QDP_Subset QDP_all, QDP_even, QDP_odd, QDP_even_and_odd[2];
extern QDP_Shift QDP_neighbor[4];
extern int QDP_this_node;
#define QDP_all_L(lat) QDP_all

/* fields: a pointer to V site values */
#define QDP_SHIM_FIELD_TYPES(PC, QPC)                                  \
  typedef struct { QLA_##QPC##_ColorVector *d; } QDP_##PC##_ColorVector; \
  typedef struct { QLA_##QPC##_ColorMatrix *d; } QDP_##PC##_ColorMatrix; \
  typedef struct { QLA_##QPC##_DiracFermion *d; } QDP_##PC##_DiracFermion; \
  typedef struct { QLA_##QPC##_HalfFermion *d; } QDP_##PC##_HalfFermion; \
  typedef struct { QLA_##QPC##_DiracPropagator *d; } QDP_##PC##_DiracPropagator;
QDP_SHIM_FIELD_TYPES(F1, F1)
QDP_SHIM_FIELD_TYPES(D1, D1)
QDP_SHIM_FIELD_TYPES(F2, F2)
QDP_SHIM_FIELD_TYPES(D2, D2)
QDP_SHIM_FIELD_TYPES(F3, F3)
QDP_SHIM_FIELD_TYPES(D3, D3)
QDP_SHIM_FIELD_TYPES(FN, FN)
QDP_SHIM_FIELD_TYPES(DN, DN)
typedef QDP_FN_ColorVector QDP_N_ColorVector;
typedef struct { QLA_F_Complex *d; } QDP_F_Complex;
typedef struct { QLA_D_Complex *d; } QDP_D_Complex;
typedef struct { QLA_F_Real *d; } QDP_F_Real;
typedef struct { QLA_D_Real *d; } QDP_D_Real;
typedef struct { int *d; } QDP_Int;

/* the API for one precision (PC = F3 or D3, P = F or D) */
#define QDP_SHIM_DECLARE(PC, P)                                                                                  \
  QDP_##PC##_ColorVector *QDP_##PC##_create_V(void);                                                            \
  void QDP_##PC##_destroy_V(QDP_##PC##_ColorVector *);                                                          \
  QDP_##PC##_ColorMatrix *QDP_##PC##_create_M(void);                                                            \
  void QDP_##PC##_destroy_M(QDP_##PC##_ColorMatrix *);                                                          \
  QDP_##P##_Complex *QDP_##P##_create_C(void);                                                                  \
  void QDP_##P##_destroy_C(QDP_##P##_Complex *);                                                                \
  QLA_##PC##_ColorVector *QDP_##PC##_expose_V(QDP_##PC##_ColorVector *);                                        \
  void QDP_##PC##_reset_V(QDP_##PC##_ColorVector *);                                                            \
  QLA_##PC##_ColorMatrix *QDP_##PC##_expose_M(QDP_##PC##_ColorMatrix *);                                        \
  void QDP_##PC##_reset_M(QDP_##PC##_ColorMatrix *);                                                            \
  void QDP_##PC##_insert_V(QDP_##PC##_ColorVector *, QLA_##PC##_ColorVector *, QDP_Subset);                     \
  void QDP_##PC##_extract_V(QLA_##PC##_ColorVector *, QDP_##PC##_ColorVector *, QDP_Subset);                    \
  void QDP_##PC##_insert_M(QDP_##PC##_ColorMatrix *, QLA_##PC##_ColorMatrix *, QDP_Subset);                     \
  void QDP_##PC##_extract_M(QLA_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *, QDP_Subset);                    \
  void QDP_##PC##_V_eq_zero(QDP_##PC##_ColorVector *, QDP_Subset);                                              \
  void QDP_##PC##_V_eq_V(QDP_##PC##_ColorVector *, QDP_##PC##_ColorVector *, QDP_Subset);                       \
  void QDP_##PC##_V_peq_V(QDP_##PC##_ColorVector *, QDP_##PC##_ColorVector *, QDP_Subset);                      \
  void QDP_##PC##_V_meq_V(QDP_##PC##_ColorVector *, QDP_##PC##_ColorVector *, QDP_Subset);                      \
  void QDP_##PC##_V_eq_V_plus_V(QDP_##PC##_ColorVector *, QDP_##PC##_ColorVector *, QDP_##PC##_ColorVector *,   \
                                QDP_Subset);                                                                     \
  void QDP_##PC##_V_eq_V_minus_V(QDP_##PC##_ColorVector *, QDP_##PC##_ColorVector *, QDP_##PC##_ColorVector *,  \
                                 QDP_Subset);                                                                    \
  void QDP_##PC##_V_eq_r_times_V(QDP_##PC##_ColorVector *, QLA_##P##_Real *, QDP_##PC##_ColorVector *,          \
                                 QDP_Subset);                                                                    \
  void QDP_##PC##_V_peq_r_times_V(QDP_##PC##_ColorVector *, QLA_##P##_Real *, QDP_##PC##_ColorVector *,         \
                                  QDP_Subset);                                                                   \
  void QDP_##PC##_V_meq_r_times_V(QDP_##PC##_ColorVector *, QLA_##P##_Real *, QDP_##PC##_ColorVector *,         \
                                  QDP_Subset);                                                                   \
  void QDP_##PC##_V_eq_r_times_V_plus_V(QDP_##PC##_ColorVector *, QLA_##P##_Real *, QDP_##PC##_ColorVector *,   \
                                        QDP_##PC##_ColorVector *, QDP_Subset);                                   \
  void QDP_##PC##_V_eq_r_times_V_minus_V(QDP_##PC##_ColorVector *, QLA_##P##_Real *, QDP_##PC##_ColorVector *,  \
                                         QDP_##PC##_ColorVector *, QDP_Subset);                                  \
  void QDP_##PC##_V_eq_c_times_V(QDP_##PC##_ColorVector *, QLA_##P##_Complex *, QDP_##PC##_ColorVector *,       \
                                 QDP_Subset);                                                                    \
  void QDP_##PC##_V_peq_c_times_V(QDP_##PC##_ColorVector *, QLA_##P##_Complex *, QDP_##PC##_ColorVector *,      \
                                  QDP_Subset);                                                                   \
  void QDP_##PC##_V_meq_c_times_V(QDP_##PC##_ColorVector *, QLA_##P##_Complex *, QDP_##PC##_ColorVector *,      \
                                  QDP_Subset);                                                                   \
  void QDP_##PC##_V_eq_c_times_V_plus_V(QDP_##PC##_ColorVector *, QLA_##P##_Complex *, QDP_##PC##_ColorVector *,\
                                        QDP_##PC##_ColorVector *, QDP_Subset);                                   \
  void QDP_##PC##_V_veq_zero(QDP_##PC##_ColorVector **, QDP_Subset, int);                                       \
  void QDP_##PC##_V_veq_V(QDP_##PC##_ColorVector **, QDP_##PC##_ColorVector **, QDP_Subset, int);               \
  void QDP_##PC##_V_vpeq_V(QDP_##PC##_ColorVector **, QDP_##PC##_ColorVector **, QDP_Subset, int);              \
  void QDP_##PC##_V_vmeq_V(QDP_##PC##_ColorVector **, QDP_##PC##_ColorVector **, QDP_Subset, int);              \
  void QDP_##PC##_V_veq_V_plus_V(QDP_##PC##_ColorVector **, QDP_##PC##_ColorVector **,                         \
                                 QDP_##PC##_ColorVector **, QDP_Subset, int);                                    \
  void QDP_##PC##_V_veq_V_minus_V(QDP_##PC##_ColorVector **, QDP_##PC##_ColorVector **,                        \
                                  QDP_##PC##_ColorVector **, QDP_Subset, int);                                   \
  void QDP_##PC##_V_veq_r_times_V(QDP_##PC##_ColorVector **, QLA_##P##_Real *, QDP_##PC##_ColorVector **,       \
                                  QDP_Subset, int);                                                              \
  void QDP_##PC##_V_vpeq_r_times_V(QDP_##PC##_ColorVector **, QLA_##P##_Real *, QDP_##PC##_ColorVector **,      \
                                   QDP_Subset, int);                                                             \
  void QDP_##PC##_V_vmeq_r_times_V(QDP_##PC##_ColorVector **, QLA_##P##_Real *, QDP_##PC##_ColorVector **,      \
                                   QDP_Subset, int);                                                             \
  void QDP_##PC##_V_vpeq_c_times_V(QDP_##PC##_ColorVector **, QLA_##P##_Complex *, QDP_##PC##_ColorVector **,   \
                                   QDP_Subset, int);                                                             \
  void QDP_##PC##_V_veq_r_times_V_plus_V(QDP_##PC##_ColorVector **, QLA_##P##_Real *,                          \
                                         QDP_##PC##_ColorVector **, QDP_##PC##_ColorVector **, QDP_Subset, int); \
  void QDP_##PC##_V_veq_c_times_V_plus_V(QDP_##PC##_ColorVector **, QLA_##P##_Complex *,                       \
                                         QDP_##PC##_ColorVector **, QDP_##PC##_ColorVector **, QDP_Subset, int); \
  void QDP_##PC##_V_veq_sV(QDP_##PC##_ColorVector **, QDP_##PC##_ColorVector **, QDP_Shift *, QDP_ShiftDir *,   \
                           QDP_Subset, int);                                                                     \
  void QDP_##PC##_V_eq_sV(QDP_##PC##_ColorVector *, QDP_##PC##_ColorVector *, QDP_Shift, QDP_ShiftDir,          \
                          QDP_Subset);                                                                           \
  void QDP_##PC##_V_vpeq_M_times_V(QDP_##PC##_ColorVector **, QDP_##PC##_ColorMatrix **,                       \
                                   QDP_##PC##_ColorVector **, QDP_Subset, int);                                  \
  void QDP_##PC##_V_veq_Ma_times_V(QDP_##PC##_ColorVector **, QDP_##PC##_ColorMatrix **,                       \
                                   QDP_##PC##_ColorVector **, QDP_Subset, int);                                  \
  void QDP_##PC##_r_eq_norm2_V(QLA_##P##_Real *, QDP_##PC##_ColorVector *, QDP_Subset);                         \
  void QDP_##PC##_r_veq_norm2_V(QLA_##P##_Real *, QDP_##PC##_ColorVector **, QDP_Subset, int);                  \
  void QDP_##PC##_r_eq_re_V_dot_V(QLA_##P##_Real *, QDP_##PC##_ColorVector *, QDP_##PC##_ColorVector *,         \
                                  QDP_Subset);                                                                   \
  void QDP_##PC##_r_veq_re_V_dot_V(QLA_##P##_Real *, QDP_##PC##_ColorVector **, QDP_##PC##_ColorVector **,      \
                                   QDP_Subset, int);                                                             \
  void QDP_##PC##_c_eq_V_dot_V(QLA_##P##_Complex *, QDP_##PC##_ColorVector *, QDP_##PC##_ColorVector *,         \
                               QDP_Subset);                                                                      \
  void QDP_##PC##_c_veq_V_dot_V(QLA_##P##_Complex *, QDP_##PC##_ColorVector **, QDP_##PC##_ColorVector **,      \
                                QDP_Subset, int);                                                                \
  void QDP_##PC##_M_eq_zero(QDP_##PC##_ColorMatrix *, QDP_Subset);                                              \
  void QDP_##PC##_M_eq_M(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *, QDP_Subset);                       \
  void QDP_##PC##_M_peq_M(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *, QDP_Subset);                      \
  void QDP_##PC##_M_eqm_Ma(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *, QDP_Subset);                     \
  void QDP_##PC##_M_eq_r_times_M(QDP_##PC##_ColorMatrix *, QLA_##P##_Real *, QDP_##PC##_ColorMatrix *,          \
                                 QDP_Subset);                                                                    \
  void QDP_##PC##_M_peq_r_times_M(QDP_##PC##_ColorMatrix *, QLA_##P##_Real *, QDP_##PC##_ColorMatrix *,         \
                                  QDP_Subset);                                                                   \
  void QDP_##PC##_M_eq_C_times_M(QDP_##PC##_ColorMatrix *, QDP_##P##_Complex *, QDP_##PC##_ColorMatrix *,       \
                                 QDP_Subset);                                                                    \
  void QDP_##PC##_M_eq_M_times_M(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *,  \
                                 QDP_Subset);                                                                    \
  void QDP_##PC##_M_eq_M_times_Ma(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *,                          \
                                  QDP_##PC##_ColorMatrix *, QDP_Subset);                                         \
  void QDP_##PC##_M_eq_Ma_times_M(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *,                          \
                                  QDP_##PC##_ColorMatrix *, QDP_Subset);                                         \
  void QDP_##PC##_M_eq_sM(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *, QDP_Shift, QDP_ShiftDir,          \
                          QDP_Subset);                                                                           \
  void QDP_##PC##_M_eq_funct(QDP_##PC##_ColorMatrix *, void (*)(QLA_##PC##_ColorMatrix *, int[]), QDP_Subset);  \
  void QDP_##PC##_r_eq_norm2_M(QLA_##P##_Real *, QDP_##PC##_ColorMatrix *, QDP_Subset);                         \
  void QDP_##PC##_m_eq_sum_M(QLA_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *, QDP_Subset);                   \
  void QDP_##P##_C_eq_c(QDP_##P##_Complex *, QLA_##P##_Complex *, QDP_Subset);                                \
  void QDP_##PC##_V_eq_funcit(QDP_##PC##_ColorVector *, void (*)(QLA_##PC##_ColorVector *, int), QDP_Subset);  \
  QDP_##PC##_DiracFermion *QDP_##PC##_create_D(void);                                                          \
  void QDP_##PC##_destroy_D(QDP_##PC##_DiracFermion *);                                                        \
  void QDP_##PC##_D_eq_D(QDP_##PC##_DiracFermion *, QDP_##PC##_DiracFermion *, QDP_Subset);                    \
  void QDP_##PC##_insert_D(QDP_##PC##_DiracFermion *, QLA_##PC##_DiracFermion *, QDP_Subset);                  \
  void QDP_##PC##_extract_D(QLA_##PC##_DiracFermion *, QDP_##PC##_DiracFermion *, QDP_Subset);                 \
  void QDP_##PC##_M_eq_Ma(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *, QDP_Subset);                      \
  void QDP_##PC##_M_peq_Ma(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *, QDP_Subset);                     \
  void QDP_##PC##_M_eqm_M(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *, QDP_Subset);                      \
  void QDP_##PC##_M_meq_M(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *, QDP_Subset);                      \
  void QDP_##PC##_M_eq_antiherm_M(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *, QDP_Subset);              \
  void QDP_##PC##_M_eq_r_times_M_plus_M(QDP_##PC##_ColorMatrix *, QLA_##P##_Real *, QDP_##PC##_ColorMatrix *,   \
                                        QDP_##PC##_ColorMatrix *, QDP_Subset);                                   \
  void QDP_##PC##_M_eq_Ma_times_Ma(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *,                         \
                                   QDP_##PC##_ColorMatrix *, QDP_Subset);                                        \
  void QDP_##PC##_M_peq_M_times_M(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *,                          \
                                  QDP_##PC##_ColorMatrix *, QDP_Subset);                                         \
  void QDP_##PC##_M_meq_M_times_M(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *,                          \
                                  QDP_##PC##_ColorMatrix *, QDP_Subset);                                         \
  void QDP_##PC##_M_peq_M_times_Ma(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorMatrix *,                         \
                                   QDP_##PC##_ColorMatrix *, QDP_Subset);                                        \
  void QDP_##PC##_M_eq_V_times_Va(QDP_##PC##_ColorMatrix *, QDP_##PC##_ColorVector *,                          \
                                  QDP_##PC##_ColorVector *, QDP_Subset);                                         \
  void QDP_##PC##_M_vpeq_V_times_Va(QDP_##PC##_ColorMatrix **, QDP_##PC##_ColorVector **,                      \
                                    QDP_##PC##_ColorVector **, QDP_Subset, int);                                 \
  void QDP_##PC##_V_veq_M_times_V(QDP_##PC##_ColorVector **, QDP_##PC##_ColorMatrix **,                        \
                                  QDP_##PC##_ColorVector **, QDP_Subset, int);
QDP_SHIM_DECLARE(F3, F)
QDP_SHIM_DECLARE(D3, D)

/* conversions between precisions */
void QDP_FD_V_eq_V(QDP_F3_ColorVector *, QDP_D3_ColorVector *, QDP_Subset);
void QDP_DF_V_eq_V(QDP_D3_ColorVector *, QDP_F3_ColorVector *, QDP_Subset);
void QDP_FD_M_eq_M(QDP_F3_ColorMatrix *, QDP_D3_ColorMatrix *, QDP_Subset);
void QDP_DF_M_eq_M(QDP_D3_ColorMatrix *, QDP_F3_ColorMatrix *, QDP_Subset);

/* lattice, layout, node (qdp_shim.c) */
extern int QDP_shim_V;                 /* sites */
extern int (*QDP_shim_coords)[4];      /* coordinates of each site */
int QDP_is_initialized(void);
int QDP_initialize(int *argc, char ***argv);
void QDP_finalize(void);
void QDP_abort(int status);
void QDP_set_default_layout(QDP_Layout *layout);
void QDP_set_latsize(int nd, int *size);
void QDP_create_layout(void);
void QDP_set_block_size(int bs);
int QDP_ndim(void);
void QDP_latsize(int *ls);
int QDP_coord_size(int i);
int QDP_volume(void);
int QDP_sites_on_node_fn(void);
#define QDP_sites_on_node QDP_sites_on_node_fn()
#define QDP_ndim_L(lat) QDP_ndim()
#define QDP_latsize_L(lat, ls) QDP_latsize(ls)
int QDP_subset_len(QDP_Subset s);
int QDP_node_number(const int x[]);
int QDP_index(const int x[]);
void QDP_get_coords(int x[], int node, int index);
QDP_Shift QDP_create_shift(int disp[]);
void QDP_destroy_shift(QDP_Shift s);
double QDP_time(void);
int QDP_profcontrol(int level);
int QDP_verbose(int level);
QDP_Lattice *QDP_get_default_lattice(void);
QDP_Subset *QDP_create_subset_L(QDP_Lattice *lat, int (*func)(QDP_Lattice *, int x[], void *), void *args,
                                int argsize, int n);

/* generic names for the precision and colours of the including unit */
#if defined(QDP_Precision) && QDP_Precision == 'F'
#define QDP_SHIM_P(x) QDP_F3_##x
#define QDP_SHIM_R(x) QDP_F_##x
#else
#define QDP_SHIM_P(x) QDP_D3_##x
#define QDP_SHIM_R(x) QDP_D_##x
#endif
#define QDP_Nc 3
#define QDP_get_nc(x) 3
#define QDP_get_lattice_V(x) ((QDP_Lattice *)0)
#define QDP_get_lattice_M(x) ((QDP_Lattice *)0)
#define QDP_discard_V(x) ((void)(x))
#define QDP_discard_M(x) ((void)(x))
#define QDP_thread_barrier() ((void)0)
/* reached only by the reference's projection for Nc != 3 */
#define QDP_M_eq_funciat(r, f, args, sub)                                  \
  do {                                                                     \
    QDP_abort(1);                                                          \
  } while (0)
typedef QDP_SHIM_P(ColorVector) QDP_ColorVector;
typedef QDP_SHIM_P(ColorMatrix) QDP_ColorMatrix;
typedef QDP_SHIM_P(DiracFermion) QDP_DiracFermion;
typedef QDP_SHIM_P(DiracPropagator) QDP_DiracPropagator;
typedef QDP_SHIM_R(Complex) QDP_Complex;
typedef QDP_SHIM_R(Real) QDP_Real;
typedef QDP_F3_ColorVector QDP_F_ColorVector;
typedef QDP_F3_ColorMatrix QDP_F_ColorMatrix;
typedef QDP_F3_DiracFermion QDP_F_DiracFermion;
typedef QDP_D3_ColorVector QDP_D_ColorVector;
typedef QDP_D3_ColorMatrix QDP_D_ColorMatrix;
typedef QDP_D3_DiracFermion QDP_D_DiracFermion;
#define QDP_F_create_V QDP_F3_create_V
#define QDP_F_destroy_V QDP_F3_destroy_V
#define QDP_F_create_M QDP_F3_create_M
#define QDP_F_destroy_M QDP_F3_destroy_M
#define QDP_D_create_V QDP_D3_create_V
#define QDP_D_destroy_V QDP_D3_destroy_V
#define QDP_D_create_M QDP_D3_create_M
#define QDP_D_destroy_M QDP_D3_destroy_M
#define QDP_F_M_eq_r_times_M QDP_F3_M_eq_r_times_M
#define QDP_D_M_eq_r_times_M QDP_D3_M_eq_r_times_M
#define QDP_F_M_eq_M QDP_F3_M_eq_M
#define QDP_D_M_eq_M QDP_D3_M_eq_M
#define QDP_F_V_eq_V QDP_F3_V_eq_V
#define QDP_D_V_eq_V QDP_D3_V_eq_V

#define QDP_create_V QDP_SHIM_P(create_V)
#define QDP_destroy_V QDP_SHIM_P(destroy_V)
#define QDP_create_M QDP_SHIM_P(create_M)
#define QDP_destroy_M QDP_SHIM_P(destroy_M)
#define QDP_create_C QDP_SHIM_R(create_C)
#define QDP_destroy_C QDP_SHIM_R(destroy_C)
#define QDP_expose_V QDP_SHIM_P(expose_V)
#define QDP_reset_V QDP_SHIM_P(reset_V)
#define QDP_expose_M QDP_SHIM_P(expose_M)
#define QDP_reset_M QDP_SHIM_P(reset_M)
#define QDP_insert_V QDP_SHIM_P(insert_V)
#define QDP_extract_V QDP_SHIM_P(extract_V)
#define QDP_insert_M QDP_SHIM_P(insert_M)
#define QDP_extract_M QDP_SHIM_P(extract_M)
#define QDP_V_eq_zero QDP_SHIM_P(V_eq_zero)
#define QDP_V_eq_V QDP_SHIM_P(V_eq_V)
#define QDP_V_peq_V QDP_SHIM_P(V_peq_V)
#define QDP_V_meq_V QDP_SHIM_P(V_meq_V)
#define QDP_V_eq_V_plus_V QDP_SHIM_P(V_eq_V_plus_V)
#define QDP_V_eq_V_minus_V QDP_SHIM_P(V_eq_V_minus_V)
#define QDP_V_eq_r_times_V QDP_SHIM_P(V_eq_r_times_V)
#define QDP_V_peq_r_times_V QDP_SHIM_P(V_peq_r_times_V)
#define QDP_V_meq_r_times_V QDP_SHIM_P(V_meq_r_times_V)
#define QDP_V_eq_r_times_V_plus_V QDP_SHIM_P(V_eq_r_times_V_plus_V)
#define QDP_V_eq_r_times_V_minus_V QDP_SHIM_P(V_eq_r_times_V_minus_V)
#define QDP_V_eq_c_times_V QDP_SHIM_P(V_eq_c_times_V)
#define QDP_V_peq_c_times_V QDP_SHIM_P(V_peq_c_times_V)
#define QDP_V_meq_c_times_V QDP_SHIM_P(V_meq_c_times_V)
#define QDP_V_eq_c_times_V_plus_V QDP_SHIM_P(V_eq_c_times_V_plus_V)
#define QDP_V_veq_zero QDP_SHIM_P(V_veq_zero)
#define QDP_V_veq_V QDP_SHIM_P(V_veq_V)
#define QDP_V_vpeq_V QDP_SHIM_P(V_vpeq_V)
#define QDP_V_vmeq_V QDP_SHIM_P(V_vmeq_V)
#define QDP_V_veq_V_plus_V QDP_SHIM_P(V_veq_V_plus_V)
#define QDP_V_veq_V_minus_V QDP_SHIM_P(V_veq_V_minus_V)
#define QDP_V_veq_r_times_V QDP_SHIM_P(V_veq_r_times_V)
#define QDP_V_vpeq_r_times_V QDP_SHIM_P(V_vpeq_r_times_V)
#define QDP_V_vmeq_r_times_V QDP_SHIM_P(V_vmeq_r_times_V)
#define QDP_V_vpeq_c_times_V QDP_SHIM_P(V_vpeq_c_times_V)
#define QDP_V_veq_r_times_V_plus_V QDP_SHIM_P(V_veq_r_times_V_plus_V)
#define QDP_V_veq_c_times_V_plus_V QDP_SHIM_P(V_veq_c_times_V_plus_V)
#define QDP_V_veq_sV QDP_SHIM_P(V_veq_sV)
#define QDP_V_eq_sV QDP_SHIM_P(V_eq_sV)
#define QDP_V_vpeq_M_times_V QDP_SHIM_P(V_vpeq_M_times_V)
#define QDP_V_veq_Ma_times_V QDP_SHIM_P(V_veq_Ma_times_V)
#define QDP_r_eq_norm2_V QDP_SHIM_P(r_eq_norm2_V)
#define QDP_r_veq_norm2_V QDP_SHIM_P(r_veq_norm2_V)
#define QDP_r_eq_re_V_dot_V QDP_SHIM_P(r_eq_re_V_dot_V)
#define QDP_r_veq_re_V_dot_V QDP_SHIM_P(r_veq_re_V_dot_V)
#define QDP_c_eq_V_dot_V QDP_SHIM_P(c_eq_V_dot_V)
#define QDP_c_veq_V_dot_V QDP_SHIM_P(c_veq_V_dot_V)
#define QDP_M_eq_zero QDP_SHIM_P(M_eq_zero)
#define QDP_M_eq_M QDP_SHIM_P(M_eq_M)
#define QDP_M_peq_M QDP_SHIM_P(M_peq_M)
#define QDP_M_eqm_Ma QDP_SHIM_P(M_eqm_Ma)
#define QDP_M_eq_r_times_M QDP_SHIM_P(M_eq_r_times_M)
#define QDP_M_peq_r_times_M QDP_SHIM_P(M_peq_r_times_M)
#define QDP_M_eq_C_times_M QDP_SHIM_P(M_eq_C_times_M)
#define QDP_M_eq_M_times_M QDP_SHIM_P(M_eq_M_times_M)
#define QDP_M_eq_M_times_Ma QDP_SHIM_P(M_eq_M_times_Ma)
#define QDP_M_eq_Ma_times_M QDP_SHIM_P(M_eq_Ma_times_M)
#define QDP_M_eq_sM QDP_SHIM_P(M_eq_sM)
#define QDP_M_eq_funct QDP_SHIM_P(M_eq_funct)
#define QDP_r_eq_norm2_M QDP_SHIM_P(r_eq_norm2_M)
#define QDP_m_eq_sum_M QDP_SHIM_P(m_eq_sum_M)
#define QDP_C_eq_c QDP_SHIM_R(C_eq_c)
#define QDP_V_eq_funcit QDP_SHIM_P(V_eq_funcit)
#define QDP_create_D QDP_SHIM_P(create_D)
#define QDP_destroy_D QDP_SHIM_P(destroy_D)
#define QDP_D_eq_D QDP_SHIM_P(D_eq_D)
#define QDP_insert_D QDP_SHIM_P(insert_D)
#define QDP_extract_D QDP_SHIM_P(extract_D)
#define QDP_M_eq_Ma QDP_SHIM_P(M_eq_Ma)
#define QDP_M_peq_Ma QDP_SHIM_P(M_peq_Ma)
#define QDP_M_eqm_M QDP_SHIM_P(M_eqm_M)
#define QDP_M_meq_M QDP_SHIM_P(M_meq_M)
#define QDP_M_eq_antiherm_M QDP_SHIM_P(M_eq_antiherm_M)
#define QDP_M_eq_r_times_M_plus_M QDP_SHIM_P(M_eq_r_times_M_plus_M)
#define QDP_M_eq_Ma_times_Ma QDP_SHIM_P(M_eq_Ma_times_Ma)
#define QDP_M_peq_M_times_M QDP_SHIM_P(M_peq_M_times_M)
#define QDP_M_meq_M_times_M QDP_SHIM_P(M_meq_M_times_M)
#define QDP_M_peq_M_times_Ma QDP_SHIM_P(M_peq_M_times_Ma)
#define QDP_M_eq_V_times_Va QDP_SHIM_P(M_eq_V_times_Va)
#define QDP_M_vpeq_V_times_Va QDP_SHIM_P(M_vpeq_V_times_Va)
#define QDP_V_veq_M_times_V QDP_SHIM_P(V_veq_M_times_V)

#ifdef __cplusplus
}
#endif
#endif
