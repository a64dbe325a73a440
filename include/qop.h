/*
 * qop.h -- drop-in C interface of the B200 asqtad/HISQ staggered library.
 *
 * A program written against QOPQDP's asqtad/HISQ API (Nc = 3, single and
 * double precision) compiles against this header unchanged and links
 * against libqop_b200.so instead of libqopqdp + QDP + QLA + QMP.
 *
 * ABI contract.  Every struct, enum and macro below has the same members,
 * order and values as the reference's include/qop_int.h, so that a caller's
 * existing structs are bit-compatible.  Handles are opaque pointers whose
 * storage lives in GPU memory.  Raw fields keep the reference's layout:
 *   ColorVector raw  : V sites x 3 colours x (re,im)         (QLA_ColorVector)
 *   ColorMatrix raw  : V sites x 3 x 3 x (re,im), row major  (QLA_ColorMatrix)
 *   site order       : even sites first, then odd; within a parity the
 *                      lexicographic index (x[0] slowest, x[3] fastest)
 *                      divided by two (lib/layout_user.c:237-258).
 *   raw arrays are always full-volume; `evenodd` selects the half that is
 *   read or written (include/qop_pc.h:28-32).
 *
 * Differences from the reference, all on the error path:
 *   - functions never call exit(); failures are returned in info->status
 *     (or as a NULL handle / QOP_FAIL return) -- reference always reported
 *     QOP_SUCCESS and aborted on errors (include/qop_internal.h:67-103);
 *   - the QDP-typed entry points (*_qdp, ddagd with QDP_ColorVector) cannot
 *     exist without QDP; ddagd / ddagd_norm2 take QOP_ColorVector handles.
 *
 * B200-only extensions live in qop_b200.h.
 */
#ifndef _QOP_H
#define _QOP_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- precision / colour selection (include/qop.h:1-100) ---------------- */
#ifndef QOP_Precision
#  ifndef QOP_PrecisionInt
#    define QOP_PrecisionInt 1
#  endif
#  if QOP_PrecisionInt == 1
#    define QOP_Precision 'F'
#  else
#    define QOP_Precision 'D'
#  endif
#endif
#ifndef QOP_Colors
#  define QOP_Colors 3
#endif
#ifndef QOP_Nc
#  define QOP_Nc 3
#endif

/* ---- scalar types and enums (include/qop_int.h:8-27) ------------------- */
#define QOP_VERB_OFF    0
#define QOP_VERB_LOW    1
#define QOP_VERB_MED    2
#define QOP_VERB_HI     3
#define QOP_VERB_DEBUG  4

typedef enum {
  QOP_SUCCESS = 0,
  QOP_FAIL = 1,
  QOP_BC_ERROR,
  QOP_MEM_ERROR,
  QOP_TOP_ERROR
} QOP_status_t;

typedef enum {
  QOP_EVEN = 0,
  QOP_ODD = 1,
  QOP_EVENODD = 2
} QOP_evenodd_t;

typedef enum {
  QOP_UNITARIZE_U3 = 0,
  QOP_UNITARIZE_SU3 = 1
} QOP_hisq_unitarize_group_t;

typedef enum {
  QOP_UNITARIZE_NONE = 0,
  QOP_UNITARIZE_RATIONAL = 3,
  QOP_UNITARIZE_ANALYTIC = 5
} QOP_hisq_unitarize_method_t;

typedef float QOP_F_Real;
typedef double QOP_D_Real;

/* ---- structs (include/qop_int.h:48-187), member order kept ------------- */
typedef struct {
  int (*node_number)(const int coords[]);
  int (*node_index)(const int coords[]);
  int latdim;
  int *latsize;
  int machdim;
  int *machsize;
  int this_node;
  int sites_on_node;
} QOP_layout_t;
#define QOP_LAYOUT_ZERO ((QOP_layout_t){NULL,NULL,0,NULL,0,NULL,0,0})

typedef struct { double re; double im; } QOP_Complex;

/* boundary phase per direction; it multiplies the last link slice */
typedef struct { QOP_Complex *phase; } QOP_bc_t;

/* staggered sign bitmask per direction: bit i set => factor (-1)^x[i] */
typedef struct { int *signmask; } QOP_staggered_sign_t;

typedef struct { char *tag; double value; void *extra; } QOP_opt_t;

typedef struct {
  double final_sec;
  double final_flop;
  QOP_status_t status;
  int count1, count2;
} QOP_info_t;
#define QOP_INFO_ZERO ((QOP_info_t){0,0,QOP_SUCCESS,0,0})

typedef struct {
  double mixed_rsq;
  int max_iter;
  int restart;
  int max_restarts;
  QOP_evenodd_t evenodd;
} QOP_invert_arg_t;
#define QOP_INVERT_ARG_DEFAULT ((QOP_invert_arg_t){1e9,2000,1000,5,QOP_EVENODD})

typedef struct {
  double rsqmin;      /* (in)  squared residual / |in|^2 target, 0 = ignore */
  double final_rsq;   /* (out) achieved squared relative residual           */
  double relmin;      /* (in)  squared Fermilab relative norm, 0 = ignore   */
  double final_rel;   /* (out)                                               */
  int final_iter;     /* (out) iterations                                    */
  int final_restart;  /* (out) restarts                                      */
} QOP_resid_arg_t;
#define QOP_RESID_ARG_DEFAULT ((QOP_resid_arg_t){1e-6,0,0,0,0,0})

typedef struct {
  double one_link;
  double three_staple;
  double five_staple;
  double seven_staple;
  double lepage;
  double naik;
} QOP_asqtad_coeffs_t;
#define QOP_ASQTAD_COEFFS_ZERO ((QOP_asqtad_coeffs_t){0,0,0,0,0,0})

#define QOP_MAX_NAIK 20
#define QOP_EPS_NAIK_ZERO {0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0}

typedef struct {
  int n_naiks;
  double eps_naik[QOP_MAX_NAIK];
  QOP_hisq_unitarize_group_t ugroup;
  QOP_hisq_unitarize_method_t umethod;
  double fat7_one_link;
  double fat7_three_staple;
  double fat7_five_staple;
  double fat7_seven_staple;
  double fat7_lepage;
  double asqtad_one_link;
  double asqtad_three_staple;
  double asqtad_five_staple;
  double asqtad_seven_staple;
  double asqtad_lepage;
  double asqtad_naik;
  double difference_one_link;
  double difference_naik;
} QOP_hisq_coeffs_t;
#define QOP_HISQ_COEFFS_ZERO \
  ((QOP_hisq_coeffs_t){1, QOP_EPS_NAIK_ZERO, QOP_UNITARIZE_U3, \
      QOP_UNITARIZE_RATIONAL, 0,0,0,0,0, 0,0,0,0,0,0, 0,0})

/* ---- general routines (include/qop_int.h:230-254) ---------------------- */
QOP_status_t QOP_init(QOP_layout_t *layout);
QOP_status_t QOP_finalize(void);
int QOP_is_initialized(void);
const char *QOP_version_str(void);
int QOP_version_int(void);
int QOP_verbose(int level);
int QOP_profcontrol(int level);
int QOP_node_number_raw(int coords[]);
int QOP_node_index_raw_V(int coords[], QOP_evenodd_t evenodd);
int QOP_node_index_raw_G(int coords[], QOP_evenodd_t evenodd);
int QOP_sites_on_node_raw_V(QOP_evenodd_t evenodd);
int QOP_sites_on_node_raw_G(QOP_evenodd_t evenodd);
QOP_status_t QOP_asqtad_invert_set_opts(QOP_opt_t opts[], int nopts);
/* fermion-force options fnmat_src_min, veclength (lib/asqtad_force.c:3-41) */
QOP_status_t QOP_asqtad_force_set_opts(QOP_opt_t opts[], int nopts);
QOP_status_t QOP_hisq_invert_set_opts(QOP_opt_t opts[], int nopts);
QOP_status_t QOP_hisq_links_set_opts(QOP_opt_t opts[], int nopts);
/* lib/hisq_force.c:29-52: fnmat_src_min (>= 0) and veclength (> 0) are
   validated and kept; force_filter (>= 0, default 5e-5) regularises the
   derivative of the U(3) projection at links whose V^+V has an eigenvalue
   below it (the derivative of V (V^+V + force_filter)^-1/2 there). */
QOP_status_t QOP_hisq_force_set_opts(QOP_opt_t opts[], int nopts);

/* ---- per precision (include/qop_f3.h / qop_d3.h) ----------------------- */
#define QOPB_DECLARE_PC(PC, REAL)                                              \
typedef struct QOP_##PC##_ColorVector_struct        QOP_##PC##_ColorVector;    \
typedef struct QOP_##PC##_GaugeField_struct         QOP_##PC##_GaugeField;     \
typedef struct QOP_##PC##_FermionLinksAsqtad_struct QOP_##PC##_FermionLinksAsqtad; \
typedef struct QOP_##PC##_FermionLinksHisq_struct   QOP_##PC##_FermionLinksHisq; \
typedef struct QOP_##PC##_Force_struct              QOP_##PC##_Force;          \
/* fields (qop_f3.h:52-66, 115) */                                             \
QOP_##PC##_ColorVector *QOP_##PC##_create_V_from_raw(REAL *src, QOP_evenodd_t evenodd); \
void QOP_##PC##_extract_V_to_raw(REAL *dest, QOP_##PC##_ColorVector *src, QOP_evenodd_t evenodd); \
void QOP_##PC##_destroy_V(QOP_##PC##_ColorVector *field);                      \
QOP_##PC##_GaugeField *QOP_##PC##_create_G_from_raw(REAL *links[], QOP_evenodd_t evenodd); \
void QOP_##PC##_extract_G_to_raw(REAL *dest[], QOP_##PC##_GaugeField *src, QOP_evenodd_t evenodd); \
void QOP_##PC##_destroy_G(QOP_##PC##_GaugeField *field);                       \
void QOP_##PC##_rephase_G(QOP_##PC##_GaugeField *links, int *r0,               \
                          QOP_bc_t *bc, QOP_staggered_sign_t *sign);           \
/* asqtad links (qop_f3.h:222-270) */                                          \
QOP_##PC##_FermionLinksAsqtad *QOP_##PC##_asqtad_create_L_from_raw(            \
    REAL *fatlinks[], REAL *longlinks[], QOP_evenodd_t evenodd);               \
QOP_##PC##_FermionLinksAsqtad *QOP_##PC##_asqtad_create_L_from_G(              \
    QOP_info_t *info, QOP_asqtad_coeffs_t *coeffs, QOP_##PC##_GaugeField *gauge); \
QOP_##PC##_FermionLinksAsqtad *QOP_##PC##_asqtad_create_L_from_G2(             \
    QOP_info_t *info, QOP_asqtad_coeffs_t *coeffs,                             \
    QOP_##PC##_GaugeField *gFat, QOP_##PC##_GaugeField *gLong);                \
void QOP_##PC##_asqtad_load_L_from_raw(QOP_##PC##_FermionLinksAsqtad *fla,     \
    REAL *fatlinks[], REAL *longlinks[], QOP_evenodd_t evenodd);               \
void QOP_##PC##_asqtad_extract_L_to_raw(REAL *fatlinks[], REAL *longlinks[],   \
    QOP_##PC##_FermionLinksAsqtad *src, QOP_evenodd_t evenodd);                \
void QOP_##PC##_asqtad_destroy_L(QOP_##PC##_FermionLinksAsqtad *field);        \
void QOP_##PC##_asqtad_rephase_L(QOP_##PC##_FermionLinksAsqtad *fla, int *r0,  \
    QOP_bc_t *bc, QOP_staggered_sign_t *sign);                                 \
/* operator (qop_f3.h:302-336) */                                              \
void QOP_##PC##_asqtad_dslash(QOP_info_t *info, QOP_##PC##_FermionLinksAsqtad *asqtad, \
    REAL mass, QOP_##PC##_ColorVector *out, QOP_##PC##_ColorVector *in,        \
    QOP_evenodd_t eo_out, QOP_evenodd_t eo_in);                                \
void QOP_##PC##_asqtad_dslash_dir(QOP_info_t *info, QOP_##PC##_FermionLinksAsqtad *asqtad, \
    int dir, int fb, double wtfat, double wtlong,                              \
    QOP_##PC##_ColorVector *out, QOP_##PC##_ColorVector *in, QOP_evenodd_t eo_out); \
void QOP_##PC##_asqtad_diaginv(QOP_info_t *info, QOP_##PC##_FermionLinksAsqtad *asqtad, \
    REAL mass, QOP_##PC##_ColorVector *out, QOP_##PC##_ColorVector *in,        \
    QOP_evenodd_t eo);                                                         \
void QOP_##PC##_asqtad_ddagd(QOP_info_t *info, QOP_##PC##_FermionLinksAsqtad *asqtad, \
    REAL mass, QOP_##PC##_ColorVector *out, QOP_##PC##_ColorVector *in,        \
    QOP_evenodd_t eo);                                                         \
REAL QOP_##PC##_asqtad_ddagd_norm2(QOP_info_t *info, QOP_##PC##_FermionLinksAsqtad *asqtad, \
    REAL mass, QOP_##PC##_ColorVector *out, QOP_##PC##_ColorVector *in,        \
    QOP_evenodd_t eo);                                                         \
/* inverters (qop_f3.h:346-371) */                                             \
void QOP_##PC##_asqtad_invert(QOP_info_t *info, QOP_##PC##_FermionLinksAsqtad *asqtad, \
    QOP_invert_arg_t *inv_arg, QOP_resid_arg_t *res_arg, REAL mass,            \
    QOP_##PC##_ColorVector *out_pt, QOP_##PC##_ColorVector *in_pt);            \
void QOP_##PC##_asqtad_invert_multi(QOP_info_t *info,                          \
    QOP_##PC##_FermionLinksAsqtad *asqtad, QOP_invert_arg_t *inv_arg,          \
    QOP_resid_arg_t **res_arg[], REAL *masses[], int nmass[],                  \
    QOP_##PC##_ColorVector **out_pt[], QOP_##PC##_ColorVector *in_pt[], int nsrc); \
/* force fields and the asqtad fermion force (qop_pc.h:53-67, 435-448) */     \
QOP_##PC##_Force *QOP_##PC##_create_F_from_raw(REAL *force[], QOP_evenodd_t evenodd); \
void QOP_##PC##_extract_F_to_raw(REAL *dest[], QOP_##PC##_Force *src, QOP_evenodd_t evenodd); \
void QOP_##PC##_destroy_F(QOP_##PC##_Force *field);                            \
void QOP_##PC##_asqtad_force(QOP_info_t *info, QOP_##PC##_GaugeField *gauge,   \
    QOP_##PC##_Force *force, QOP_asqtad_coeffs_t *coeffs, REAL eps,            \
    QOP_##PC##_ColorVector *in_pt);                                            \
void QOP_##PC##_asqtad_force_multi(QOP_info_t *info, QOP_##PC##_GaugeField *gauge, \
    QOP_##PC##_Force *force, QOP_asqtad_coeffs_t *coef, REAL eps[],            \
    QOP_##PC##_ColorVector *in_pt[], int nsrc);                                \
void QOP_##PC##_hisq_force_multi(QOP_info_t *info, QOP_##PC##_FermionLinksHisq *flh, \
    QOP_##PC##_Force *force, QOP_hisq_coeffs_t *coef, REAL eps[],              \
    QOP_##PC##_ColorVector *in_pt[], int *n_orders_naik);                      \
/* HISQ links (qop_f3.h:473-483) */                                            \
QOP_##PC##_FermionLinksHisq *QOP_##PC##_hisq_create_L_from_G(QOP_info_t *info, \
    QOP_hisq_coeffs_t *coeffs, QOP_##PC##_GaugeField *gauge);                  \
void QOP_##PC##_hisq_destroy_L(QOP_##PC##_FermionLinksHisq *field);            \
QOP_##PC##_FermionLinksAsqtad **QOP_##PC##_get_asqtad_links_from_hisq(         \
    QOP_##PC##_FermionLinksHisq *hl);                                          \
QOP_##PC##_FermionLinksAsqtad *QOP_##PC##_get_asqtad_deps_links_from_hisq(     \
    QOP_##PC##_FermionLinksHisq *hl);

QOPB_DECLARE_PC(F3, QOP_F_Real)
QOPB_DECLARE_PC(D3, QOP_D_Real)

/* mixed-precision link copy (lib/asqtad_dslash_p.c:844-854) */
QOP_F3_FermionLinksAsqtad *QOP_FD3_asqtad_create_L_from_L(QOP_D3_FermionLinksAsqtad *fla_src);

/* ---- generic names (include/qop_f3_generic.h, qop_d3_generic.h) -------- */
#if QOP_Precision == 'F'
#  define QOPB_GEN(x) QOP_F3_##x
typedef QOP_F_Real QOP_Real;
#else
#  define QOPB_GEN(x) QOP_D3_##x
typedef QOP_D_Real QOP_Real;
#endif
#define QOP_ColorVector                 QOPB_GEN(ColorVector)
#define QOP_GaugeField                  QOPB_GEN(GaugeField)
#define QOP_FermionLinksAsqtad          QOPB_GEN(FermionLinksAsqtad)
#define QOP_FermionLinksHisq            QOPB_GEN(FermionLinksHisq)
#define QOP_create_V_from_raw           QOPB_GEN(create_V_from_raw)
#define QOP_extract_V_to_raw            QOPB_GEN(extract_V_to_raw)
#define QOP_destroy_V                   QOPB_GEN(destroy_V)
#define QOP_create_G_from_raw           QOPB_GEN(create_G_from_raw)
#define QOP_Force                       QOPB_GEN(Force)
#define QOP_create_F_from_raw           QOPB_GEN(create_F_from_raw)
#define QOP_extract_F_to_raw            QOPB_GEN(extract_F_to_raw)
#define QOP_destroy_F                   QOPB_GEN(destroy_F)
#define QOP_asqtad_force                QOPB_GEN(asqtad_force)
#define QOP_asqtad_force_multi          QOPB_GEN(asqtad_force_multi)
#define QOP_hisq_force_multi            QOPB_GEN(hisq_force_multi)
#define QOP_extract_G_to_raw            QOPB_GEN(extract_G_to_raw)
#define QOP_destroy_G                   QOPB_GEN(destroy_G)
#define QOP_rephase_G                   QOPB_GEN(rephase_G)
#define QOP_asqtad_create_L_from_raw    QOPB_GEN(asqtad_create_L_from_raw)
#define QOP_asqtad_create_L_from_G      QOPB_GEN(asqtad_create_L_from_G)
#define QOP_asqtad_create_L_from_G2     QOPB_GEN(asqtad_create_L_from_G2)
#define QOP_asqtad_load_L_from_raw      QOPB_GEN(asqtad_load_L_from_raw)
#define QOP_asqtad_extract_L_to_raw     QOPB_GEN(asqtad_extract_L_to_raw)
#define QOP_asqtad_destroy_L            QOPB_GEN(asqtad_destroy_L)
#define QOP_asqtad_rephase_L            QOPB_GEN(asqtad_rephase_L)
#define QOP_asqtad_dslash               QOPB_GEN(asqtad_dslash)
#define QOP_asqtad_dslash_dir           QOPB_GEN(asqtad_dslash_dir)
#define QOP_asqtad_diaginv              QOPB_GEN(asqtad_diaginv)
#define QOP_asqtad_ddagd                QOPB_GEN(asqtad_ddagd)
#define QOP_asqtad_ddagd_norm2          QOPB_GEN(asqtad_ddagd_norm2)
#define QOP_asqtad_invert               QOPB_GEN(asqtad_invert)
#define QOP_asqtad_invert_multi         QOPB_GEN(asqtad_invert_multi)
#define QOP_hisq_create_L_from_G        QOPB_GEN(hisq_create_L_from_G)
#define QOP_hisq_destroy_L              QOPB_GEN(hisq_destroy_L)
#define QOP_get_asqtad_links_from_hisq  QOPB_GEN(get_asqtad_links_from_hisq)
#define QOP_get_asqtad_deps_links_from_hisq QOPB_GEN(get_asqtad_deps_links_from_hisq)

#ifdef __cplusplus
}
#endif

#endif /* _QOP_H */
