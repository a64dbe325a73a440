// noalloc.cu -- QOPB_D3_asqtad_ddagd_norm2_noalloc: the normal-equation
// operator A = m^2 - D_eo D_oe with |D_oe in|^2 + m^2 |in|^2, computed
// without any device allocation.  It has no counterpart in the reference.
//
// Who needs it: callers that cannot allocate device memory at the point
// where they apply the operator.  Applications with their own caching
// allocator (a lattice code's memory manager, a framework's pool) often
// reserve nearly all of the GPU's memory up front, so a cudaMalloc from this
// library fails there even though the application has room; and inner loops
// that must not stall on the allocator (cudaMalloc and a first-fit pool
// growth can synchronise the device) want the operator with no allocation at
// all.  The regular QOP_D3_asqtad_ddagd_norm2 allocates a temporary parity
// vector per call.
//
// Scratch: one file-scope __device__ array of NOALLOC_MAX_VH * 48 bytes plus
// the reduction partials, the completion ticket and two result doubles
// (about 3.2 MB; every GPU that loads the library holds it until exit).
// Lattices with more than NOALLOC_MAX_VH sites per parity are rejected.
// Every call shares the array and leaves its contents behind; the ticket is
// cleared at the start of each call.  Calls that overlap on the GPU (for
// example from several host threads or streams) race on the array.
//
// The first call on a device looks up the array's device address (the host
// symbol is only a stand-in) with that device current; the lookup is
// guarded by a lock, so first calls from several host threads are safe.
// That first call should come before any stream capture begins.  The call
// is synchronous: it waits on the library stream and returns the norm to
// the host.
#include "qopb.h"
#include <mutex>

namespace qopb {

constexpr i64 NOALLOC_MAX_VH = 65536;                 // sites per parity (e.g. 16^4 = 2 x 32768)
constexpr i64 NOALLOC_TMP = 6 * NOALLOC_MAX_VH;       // one parity block [3][Vh] of double2, in doubles
constexpr i64 NOALLOC_PART = NOALLOC_MAX_VH / 64;     // >= one partial per 128-thread block
constexpr i64 NOALLOC_DOUBLES = NOALLOC_TMP + NOALLOC_PART + 8;

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];

// device address of the scratch array, looked up once per device with that
// device current (the host-side symbol is only a stand-in, not an address)
static double *g_scratch_dev[64];
static std::mutex g_scratch_mu;

static double *scratch_for_current_device() {
  int dev = 0;
  QCHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) fail(QOP_FAIL, "noalloc: device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_dev[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      fail(QOP_FAIL, "noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
    }
    g_scratch_dev[dev] = (double *)p;
  }
  return g_scratch_dev[dev];
}

}  // namespace qopb

using namespace qopb;

extern "C" double QOPB_D3_asqtad_ddagd_norm2_noalloc(QOP_info_t *info, QOP_D3_FermionLinksAsqtad *asqtad, double mass,
                                                     QOP_D3_ColorVector *out, QOP_D3_ColorVector *in,
                                                     QOP_evenodd_t eo) {
  try {
    require_init("QOPB_D3_asqtad_ddagd_norm2_noalloc");
    dd_refuse("QOPB_D3_asqtad_ddagd_norm2_noalloc");
    // live handles of the current lattice only: their arrays are indexed
    // with the current lattice's Vh below
    handle_check(asqtad, "FermionLinksAsqtad");
    handle_check(out, "ColorVector");
    handle_check(in, "ColorVector");
    FlaT<double> *f = reinterpret_cast<FlaT<double> *>(asqtad);
    VecT<double> *o = reinterpret_cast<VecT<double> *>(out), *i = reinterpret_cast<VecT<double> *>(in);
    if (eo != QOP_EVEN && eo != QOP_ODD) fail(QOP_FAIL, "QOPB_D3_asqtad_ddagd_norm2_noalloc: eo must be EVEN or ODD");
    const Geom &g = ctx().g;
    if (g.Vh > NOALLOC_MAX_VH)
      fail(QOP_FAIL,
           "QOPB_D3_asqtad_ddagd_norm2_noalloc: %lld sites per parity exceed the fixed scratch of %lld; "
           "use QOP_D3_asqtad_ddagd_norm2",
           (long long)g.Vh, (long long)NOALLOC_MAX_VH);
    double *base = scratch_for_current_device();
    double2 *tmp = reinterpret_cast<double2 *>(base);
    double *part = base + NOALLOC_TMP;
    unsigned *ticket = reinterpret_cast<unsigned *>(base + NOALLOC_TMP + NOALLOC_PART);
    double *res = base + NOALLOC_TMP + NOALLOC_PART + 2;
    Context &c = ctx();
    QCHECK(cudaMemsetAsync(ticket, 0, sizeof(unsigned), c.s));
    Dslash<double>::ddagd_norm2_ws(f, mass, o->d, i->d, eo, tmp, part, ticket, res);
    double h[2] = {0, 0};
    QCHECK(cudaMemcpyAsync(h, res, sizeof h, cudaMemcpyDeviceToHost, c.s));
    QCHECK(cudaStreamSynchronize(c.s));
    if (info) info->status = QOP_SUCCESS;
    return h[0] + mass * mass * h[1];
  } catch (Fail &e) {
    fprintf(stderr, "%s\n", e.msg.c_str());
    if (info) info->status = e.status;
    return -1.0;
  }
}
