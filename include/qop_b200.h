/*
 * qop_b200.h -- B200-only extensions to the QOP interface (qop.h).
 * None of these has a counterpart in the reference; a QOPQDP caller needs
 * only qop.h.  They expose what a GPU caller needs around the reference
 * API: the stream the library orders its work on, and per-kernel device
 * timings for roofline accounting.
 */
#ifndef _QOP_B200_H
#define _QOP_B200_H
#include "qop.h"
#ifdef __cplusplus
extern "C" {
#endif

/* The cudaStream_t (as void*) on which every kernel and copy of the library
   is ordered.  Valid after QOP_init.  A caller may record CUDA events on it
   to time library calls on the device. */
void *QOPB_stream(void);

/* Per-kernel-class device timing.  Between QOPB_prof_begin() and
   QOPB_prof_end() every Dslash-class launch is bracketed by CUDA events on
   the library stream.  QOPB_prof_end synchronises, fills up to `max`
   records and returns the number of kernel classes seen. */
typedef struct {
  char name[32];            /* kernel class, e.g. "hop_f16_r13"           */
  int launches;             /* launches recorded                          */
  double total_ms;          /* summed device time of those launches       */
  double bytes_per_launch;  /* mean algorithmic (compulsory) bytes per launch */
} QOPB_kstat_t;
int QOPB_prof_begin(void);
int QOPB_prof_end(QOPB_kstat_t *out, int max);
/* Bracket only launches 0, n, 2n, ... of each kernel class (n >= 1; 1, the
   default, brackets every launch).  Each pair of event records costs the
   stream a few microseconds, so sampling keeps long timed regions close to
   their unprofiled speed.  Returns 0, or -1 for n < 1. */
int QOPB_prof_every(int n);

/* Number of kernels the library has launched since it was loaded. */
unsigned long long QOPB_launch_count(void);
/* Failure injection for tests: the n-th device allocation from now on
   (n >= 1) fails as an out-of-memory would, and the call that makes it
   reports QOP_MEM_ERROR; n = 0 cancels.  Returns 0, or -1 for n < 0. */
int QOPB_inject_alloc_failure(int n);

/* QOP_D3_asqtad_ddagd_norm2 without any device allocation (no counterpart
   in the reference).  For callers that cannot allocate device memory where
   they apply the operator: applications whose own caching allocator has
   reserved nearly all of the GPU's memory (a cudaMalloc from this library
   would fail there), and loops that must not wait on an allocator.  It
   computes out = m^2 in - D_eo,oe D_oe,eo in on parity eo (QOP_EVEN or
   QOP_ODD) and returns |D_oe in|^2 + m^2 |in|^2, like the regular entry
   point; the handles must be live handles of the current lattice.  Its
   scratch is a fixed array inside the library (about 3.2 MB, held on every
   GPU that loads the library until exit), so lattices with more than 65536
   sites per parity are rejected with info->status = QOP_FAIL and a return
   value of -1.  The call is synchronous (it returns the norm to the host).
   The first call on a device looks up that array's device address under a
   lock; make that first call before any stream capture begins.  All calls
   share the array: calls that overlap on the GPU race and
   must be serialised by the caller. */
double QOPB_D3_asqtad_ddagd_norm2_noalloc(QOP_info_t *info, QOP_D3_FermionLinksAsqtad *asqtad, double mass,
                                          QOP_D3_ColorVector *out, QOP_D3_ColorVector *in, QOP_evenodd_t eo);

/* eigCG (QOP_asqtad_invert_set_opts tag "cg" = 1) keeps, in each link
   handle, one space of approximate low eigenvectors of m^2 - D_pq D_qp per
   solve parity p.  QOPB_*_eigcg_values copies up to `max` of the stored
   eigenvalues for parity eo (QOP_EVEN or QOP_ODD; ascending, at the mass of
   the last eigCG solve on that parity) into l and returns how many are
   stored: 0 before the first eigCG solve, -1 on error. */
int QOPB_F3_eigcg_values(QOP_F3_FermionLinksAsqtad *L, QOP_evenodd_t eo, double *l, int max);
int QOPB_D3_eigcg_values(QOP_D3_FermionLinksAsqtad *L, QOP_evenodd_t eo, double *l, int max);

/* Decomposed lattice, one process per GPU (the reference does this through
   QDP/QMP: lib/common.c:40-83, lib/layout_user.c:79-258).  Before QOP_init,
   rank 0 makes an NCCL id with QOPB_comm_unique_id, the host sends it to the
   other processes (e.g. through torch.distributed), and every process calls
   QOPB_comm_init(id, nranks, rank) with its GPU current.  QOP_init then
   splits the lattice as layout->machsize says (machdim 4), or, when machdim
   is <= 0, as the reference's hypercubic layout does (QOPB_layout_hyper).
   Every block must have even extents of at least 4.  Raw fields are
   node-local: QOP_sites_on_node_raw_V sites in the order of
   QOP_node_index_raw_V, and QOP_node_number_raw names the owning process.
   Dslash, dslash_dir, ddagd(_norm2), diaginv, invert, invert_multi and eigCG
   run on the decomposed lattice, with halos exchanged by NCCL on the library
   stream and reductions summed by an NCCL all-reduce.  The solvers use the
   reference algorithm there (prec_sloppy acts as 64).  Link smearing, HISQ
   links, forces, the no-alloc entry point, extra lattices and the solve
   service report QOP_FAIL (or -1).  QOPB_comm_finalize (after QOP_finalize)
   frees the communicator.  QOPB_dd_self_split(mask), called before
   QOP_init, marks directions as decomposed with this process as its own
   neighbour (halos still packed and exchanged: a one-GPU test of the
   decomposed path).  QOPB_dd_info returns this process's rank and fills the
   grid, its block coordinates, the local extents and the decomposed
   directions.  The QOPB_layout_* functions need no GPU and no QOP_init. */
int QOPB_comm_unique_id(unsigned char id[128]);
int QOPB_comm_init(const unsigned char id[128], int nranks, int rank);
int QOPB_comm_finalize(void);
int QOPB_dd_self_split(int mask);
int QOPB_dd_info(int nsquares[4], int coords[4], int local[4], int *mask);
int QOPB_layout_hyper(const int latsize[4], int nranks, int nsquares[4]);
int QOPB_layout_node_number(const int latsize[4], const int nsquares[4], const int coords[4]);
long QOPB_layout_node_index(const int latsize[4], const int nsquares[4], const int coords[4]);
int QOPB_layout_neighbors(const int nsquares[4], int rank, int nbr[8]);
/* The halo plan of the decomposed hop, for host-side checks (no GPU, no
   QOP_init).  local: the block's extents (even, >= 4).  QOPB_dd_pack_site
   gives the local site x packed into element (slab, face) of direction mu's
   halo for a parity-`parity` input (nlinks 8 or 16): the return value is -1
   for a raw slab (the input vector at x, sent to the -mu neighbour's up
   halo) or the link slot of a product slab (-U^+ psi at x with that slot's
   forward link, sent to the +mu neighbour's down halo), -2 for invalid
   arguments.  QOPB_dd_halo_ref says where the hop term (mu, disp) of local
   site x reads its neighbour: 0 inside the block, 1 the up halo, 2 the down
   halo (then *slab, *face locate the element), -1 for invalid arguments.
   Slabs hold 3 colours x fh face sites, fh = local volume / local[mu] / 2. */
int QOPB_dd_pack_site(const int local[4], int mu, int nlinks, int parity, int slab, int face, int x[4]);
int QOPB_dd_halo_ref(const int local[4], const int x[4], int mu, int disp, int *slab, int *face);

/* Several lattices in one process (no counterpart in the reference, whose
   QOP_init fixes one geometry per process).  QOP_init defines lattice 0;
   QOPB_lattice_create adds a geometry (extents even and >= 4) and returns
   its id (-1 on error); QOPB_lattice_use makes it current (0, or -1 for an
   unknown id).  Every handle belongs to the lattice that was current when it
   was created; entry points given a handle of another lattice report
   QOP_FAIL. */
int QOPB_lattice_create(const int latsize[4]);
int QOPB_lattice_use(int id);
int QOPB_lattice_current(void);

/* Solve service (no counterpart in the reference).  A worker thread keeps
   a batched mixed-precision solver (16 slots; int16 storage, FP64 reliable
   updates: every solution meets its FP64 target) per link handle and
   parity in flight and admits the systems of queued requests into free
   slots between solver steps (continuous batching); each finished system's
   result is copied to the caller's buffer.  Option tag serve_policy: 0
   steps every solver in turn (default), 1 only the one holding the oldest
   request.  A request solves, for each of its
   nrhs sources, A x = b with A = m^2 - D D on parity `evenodd` (QOP_EVEN or
   QOP_ODD) and writes m A^-1 b on that parity (the QOP_asqtad_invert
   convention) into dst[k]; src[k] / dst[k] are raw full-volume arrays
   (QOP raw site order, 6 doubles per site) that the caller keeps valid until
   QOPB_serve_wait has returned for the ticket.  While the service runs, the
   worker is the only thread that may call into the library: callers use
   only QOPB_serve_submit / QOPB_serve_wait / QOPB_serve_stop. */
typedef struct {
  QOP_D3_FermionLinksAsqtad *links; /* handle (of lattice `lattice`)        */
  int lattice;                      /* lattice id of the handle             */
  QOP_evenodd_t evenodd;            /* QOP_EVEN or QOP_ODD                  */
  double mass;
  double rsqmin;                    /* target |r|^2 / |b|^2                 */
  int max_iter;                     /* per system; <= 0: 100000             */
  int nrhs;                         /* 1 .. 16                              */
  const double *const *src;         /* nrhs raw sources                     */
  double *const *dst;               /* nrhs raw outputs                     */
} QOPB_request_t;
typedef struct {
  int status;                       /* QOP_SUCCESS or QOP_FAIL              */
  int iters_max;                    /* largest iteration count of the request */
  double final_rsq_max;             /* largest final |r|^2 / |b|^2          */
  double queue_ms, solve_ms, total_ms; /* waiting, batch solve, submit->done */
  int batch_systems;                /* systems in the batch that solved it  */
} QOPB_result_t;
int QOPB_serve_start(void);                                 /* 0 or -1 */
long long QOPB_serve_submit(const QOPB_request_t *req);     /* ticket >= 0, or -1 */
/* 0: done (result filled, ticket released); 1: timed out; -1: bad ticket */
int QOPB_serve_wait(long long ticket, double timeout_s, QOPB_result_t *res);
int QOPB_serve_stop(void);   /* finishes queued requests, joins the worker */

/* Operator checks (no counterpart in the reference).  They apply the
   reduced-precision normal-equation operator of the mixed solvers once, with
   the solvers' own kernels, so that it can be compared site by site with the
   FP64 operator QOP_D3_asqtad_ddagd_norm2 (lib/asqtad_dslash_p.c:1121-1138).
   p = int16(in) on parity eo (QOP_EVEN or QOP_ODD), t = D_oe p (written to
   t_out on the other parity), Ap = m^2 p - D_eo t (written to ap_out on
   parity eo); both are the int16 values the solver would store, decoded.
   QOPB_D3_sloppy_ddagd: one system; variant = an int16 hop variant (0..28,
   the hop_kernel option), kind2 = 2 (plain second hop) or 3 (the
   fused-update second hop, variants 20..28); sums = |t|^2, |p|^2, <p, Ap>,
   |Ap|^2 as the kernels reduced them (the last two for kind 3 only).
   QOPB_D3_sloppy_ddagd_batch: n <= 16 systems sharing the link stream;
   variant = a batch_kernel value (0..15: int16 vectors; 16: the tensor-core
   hop on bf16 hi / lo vectors) or -1 for the solver's default;
   sums[2j], sums[2j+1] = |t_j|^2 and <p_j, A_j p_j>.  Both return 0, or -1
   with info->status = QOP_FAIL. */
int QOPB_D3_sloppy_ddagd(QOP_info_t *info, QOP_D3_FermionLinksAsqtad *asqtad, double mass,
                         QOP_D3_ColorVector *t_out, QOP_D3_ColorVector *ap_out, QOP_D3_ColorVector *in,
                         QOP_evenodd_t eo, int variant, int kind2, double *sums);
int QOPB_D3_sloppy_ddagd_batch(QOP_info_t *info, QOP_D3_FermionLinksAsqtad *asqtad, int n, const double *masses,
                               QOP_D3_ColorVector **t_out, QOP_D3_ColorVector **ap_out, QOP_D3_ColorVector **in,
                               QOP_evenodd_t eo, int variant, double *sums);

#ifdef __cplusplus
}
#endif
#endif
