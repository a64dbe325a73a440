/*
 * qop_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement (plain C99 + OpenMP, FP64 throughout) of the QOPQDP
 * asqtad/HISQ hot path.  It is the parity checker for the CUDA library and
 * the timed CPU baseline; nothing in the product links or calls it.
 *
 * Parity status: pinned to the reference itself.  The reference's sources
 * need the external QDP/C, QLA and QMP libraries (absent); oracle/ref
 * supplies a single-process CPU stand-in for the calls its asqtad/HISQ path
 * makes and compiles those sources, unmodified, into
 * oracle/_ref/libqopref.so.  tests/test_ref_pin.py checks this oracle
 * against that library (links, Dslash, invert, invert_multi: rounding-level
 * agreement, equal iteration counts) and against its committed outputs in
 * tests/golden/qopref_4x4x4x4.npz.  The reference's own self-consistency
 * tests (examples/asqtad_test.c check_op, check_resids) are checked too.
 *
 * Fields are host arrays of doubles in the reference raw layout:
 *   vector  : V x 3 x (re,im)       matrix : V x 3 x 3 x (re,im)
 *   site order: even sites first, then odd (lib/layout_user.c:237-258).
 */
#ifndef QOP_ORACLE_H
#define QOP_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_lat or_lat;
typedef struct or_fla or_fla;

typedef struct {
  double mixed_rsq; int max_iter; int restart; int max_restarts; int evenodd;
} or_invert_arg;
typedef struct {
  double rsqmin, final_rsq, relmin, final_rel; int final_iter, final_restart;
} or_resid_arg;

/* lattice geometry and raw site order */
or_lat *or_lat_create(const int L[4]);
void or_lat_destroy(or_lat *g);
long or_lat_volume(const or_lat *g);
long or_raw_index(const or_lat *g, const int x[4]);
void or_raw_coords(const or_lat *g, long idx, int x[4]);
long or_neighbor(const or_lat *g, long idx, int mu, int disp);

/* gauge-field setup */
void or_rephase_G(const or_lat *g, double *links[4], const int r0[4],
                  const double *bc_reim /* 8 doubles or NULL */,
                  const int *signmask /* 4 ints or NULL */);
void or_make_imp_links(const or_lat *g, const double coef[6],
                       double *gf[4], double *gfLong[4],
                       double *fl[4], double *ll[4] /* NULL => no Naik */);
int or_u3_un_analytic(const double V[18], double W[18], int allow_svd,
                      double svd_rel_err, double svd_abs_err);
int or_u3reunit(const or_lat *g, double *Vf, double *Wf);
/* HISQ: returns number of SVD-fallback sites. out fat/long = asqtad stage
   (eps index 0); hcoef layout = 18 doubles:
   fat7[1,3,5,7,lepage], asqtad[1,3,5,7,lepage,naik], diff[1,naik],
   use_fat7_lepage, allow_svd, svd_rel, svd_abs, force_filter (the last one
   read by the force routines only) */
int or_hisq_links(const or_lat *g, const double hcoef[18], double *gauge[4],
                  double *fat[4], double *lng[4], double *W[4] /* may be NULL */);

/* asqtad operator object (links scaled by 1/2, double stored) */
or_fla *or_fla_create(or_lat *g, double *fat[4], double *lng[4] /* may be NULL */);
void or_fla_destroy(or_fla *f);
void or_dslash(or_fla *f, double mass, double *out, const double *in,
               int eo_out, int eo_in);
void or_dslash_dir(or_fla *f, int dir, int fb, double wtfat, double wtlong,
                   double *out, const double *in, int eo_out);
void or_ddagd(or_fla *f, double mass, double *out, const double *in, int eo);
double or_ddagd_norm2(or_fla *f, double mass, double *out, const double *in, int eo);
/* examples/asqtad_test.c:37-81: |chk-out|^2/|in|^2 with chk rebuilt from
   unscaled links and plain shifts */
double or_check_op(or_fla *f, double mass, const double *in,
                   double *fat[4], double *lng[4]);
double or_relnorm2(const or_lat *g, const double *r, const double *x, int eo);

/* inverters (lib/asqtad_invert_p.c) */
void or_invert(or_fla *f, or_invert_arg *ia, or_resid_arg *ra, double mass,
               double *out, const double *in, double *final_flop);
void or_invert_multi(or_fla *f, or_invert_arg *ia, or_resid_arg **ra[],
                     double *masses[], int nmass[], double **out[],
                     double *in[], int nsrc, double *final_flop);
void or_solve_multi(or_fla *f, or_invert_arg *ia, or_resid_arg *ra[],
                    double masses[], double *out[], double *in[], int nsolve,
                    double *final_flop);

/* asqtad fermion force (lib/asqtad_force_p.c:16-64, asqtad_force_fnmat_p.c).
   deriv: the derivative of
     E(U) = Re sum_{x,mu} tr[ midF_mu(x)^+ fat_mu(x) + midN_mu(x)^+ long_mu(x) ]
   with (fat, long) = make_imp_links(coef, U, U), in the convention
   dE = Re sum tr[ deriv^+ dU ]; midN may be NULL (no Naik term).
   force: the outer products midF_mu(x) = -s(x) sum_i eps_i x_i(x) x_i(x+mu)^+
   (midN with x+3mu; s = +1 even, -1 odd sites), deriv, and
   force_mu += -2 TA(U_mu deriv_mu^+), TA the traceless anti-Hermitian part
   (the FNMAT algorithm); asvec != 0 gives the reference's ASVEC result,
   force_mu = TA(force_mu) - TA(U_mu deriv_mu^+) (asqtad_force_p.c:22 picks it
   for nsrc < fnmat_src_min, 2 by default). */
/* lepage_rep != 0 adds the reference's extra Lepage term, of the form
   U_mu H with H Hermitian (asqtad_force_fnmat_p.c:316-340), giving the
   reference's own derivative field; 0 gives dE/dU for general complex U. */
void or_asqtad_deriv(const or_lat *g, const double coef[6], double *U[4],
                     double *midF[4], double *midN[4], double *deriv[4], int lepage_rep);
void or_asqtad_force(const or_lat *g, const double coef[6], double *U[4],
                     double *force[4], const double *eps, double *x[], int nsrc, int asvec);

/* HISQ fermion force (lib/hisq_force_p.c:50-80, hisq_force_fnmat2_p.c:7-231).
   W = reunit(V), V = fat7(U) (or_hisq_links).  deriv is the derivative of
     E(U) = sum_k c_k Re sum tr[ MF_k^+ fat_k(W) + MN_k^+ long_k(W) ]
   (k = 0: asqtad coefficients, c_0 = 1; k >= 1: difference coefficients,
   c_k = eps_naik[k]); mids are n_naiks x 4 fields.  The force builds
   MF_k = s(x) sum_i res_i x_i(x) x_i(x+mu)^+ over group k's sources (group 0:
   all sources; s = +1 even, -1 odd) and adds TA(U_mu (2 deriv_mu)^+).  The
   W-level derivative is the reference's field (or_asqtad_deriv with
   lepage_rep): the filtered U(3) adjoint (hcoef[17] > 0) does not remove its
   Lepage term. */
void or_hisq_deriv(const or_lat *g, const double hcoef[18], double *U[4], int n_naiks, const double *eps_naik,
                   double **midF, double **midN, double *deriv[4]);
void or_hisq_force(const or_lat *g, const double hcoef[18], double *U[4], int n_naiks, const double *eps_naik,
                   double *force[4], const double *res, double *x[], const int *n_orders_naik);

/* threads used by OpenMP regions (0 = leave default) */
void or_set_threads(int n);
int or_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
