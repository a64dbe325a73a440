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

/* Number of kernels the library has launched since it was loaded. */
unsigned long long QOPB_launch_count(void);

/* QOP_D3_asqtad_ddagd_norm2 without any device allocation (no counterpart
   in the reference).  For callers that cannot allocate device memory where
   they apply the operator: code recorded into a CUDA graph (allocation is
   not allowed during stream capture), programs whose own allocator has
   reserved the device memory, and loops that must not wait on an
   allocator.  It computes out = m^2 in - D_eo,oe D_oe,eo in on parity eo
   (QOP_EVEN or QOP_ODD) and returns |D_oe in|^2 + m^2 |in|^2, like the
   regular entry point.  Its scratch is a fixed array inside the library
   (about 3.2 MB, held on every GPU that loads the library until exit), so
   lattices with more than 65536 sites per parity are rejected with
   info->status = QOP_FAIL and a return value of -1.  The first call on a
   device looks up that array's device address; make that first call before
   any stream capture.  All calls share the array: calls that overlap on the
   GPU race and must be serialised by the caller. */
double QOPB_D3_asqtad_ddagd_norm2_noalloc(QOP_info_t *info, QOP_D3_FermionLinksAsqtad *asqtad, double mass,
                                          QOP_D3_ColorVector *out, QOP_D3_ColorVector *in, QOP_evenodd_t eo);

#ifdef __cplusplus
}
#endif
#endif
