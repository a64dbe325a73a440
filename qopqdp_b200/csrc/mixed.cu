// mixed.cu -- reduced-precision inner solves (filled in by the mixed-
// precision solver; until then every request falls back to the reference
// algorithm in FP64, which is exact).
#include "solvers.cuh"

namespace qopb {

void sloppy_invalidate(void *fla_any) { (void)fla_any; }

bool mixed_cgms(LinOp<double> &L, QOP_invert_arg_t *ia, QOP_resid_arg_t **ra, const double *shifts, int ns,
                c2<double> **out, const c2<double> *in, int eo, int prec) {
  (void)L; (void)ia; (void)ra; (void)shifts; (void)ns; (void)out; (void)in; (void)eo; (void)prec;
  return false;
}

}  // namespace qopb
