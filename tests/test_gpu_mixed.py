"""Mixed-precision reliable-update solves (prec_sloppy 16 / 32) reach the
requested FP64 true residual and agree with the FP64 oracle solve within
the accuracy the tolerance implies."""
import numpy as np
import pytest

import oracle as O
from conftest import gpu_lattice
from helpers import hisq_links, asqtad_links, eo_residual, rel_norm_err, half
from qopqdp_b200 import lattice as LT
from qopqdp_b200.qop import QOP_invert_arg_t, QOP_resid_arg_t

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [16, 32])
@pytest.mark.parametrize("L,kind,m", [((4, 4, 4, 8), "hisq", 0.05), ((8, 8, 8, 8), "asqtad", 0.02)])
def test_mixed_solve_reaches_fp64_tolerance(prec, L, kind, m):
    q = gpu_lattice(L, "D")
    V = int(np.prod(L))
    if kind == "hisq":
        fat, lng, _, _ = hisq_links(L, 0.5, 9)
    else:
        fat, lng = asqtad_links(L, 0.3, 7)
    fo = O.Fla(O.Lattice(L), fat, lng)
    fla = q.create_L_from_raw(fat, lng)
    src = LT.gaussian_vector(L, 101)
    for eo in (0, 1):
        for rsq in (1e-20, 1e-14):
            assert q.set_opts(prec_sloppy=prec) == 0
            ia = QOP_invert_arg_t(1e9, 20000, 20000, 5, eo)
            ra = QOP_resid_arg_t(rsq, 0, 0, 0, 0, 0)
            hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
            q.invert(fla, m, hout, hin, ia, ra)
            got = q.extract_V(hout, V)
            true = eo_residual(fo, m, got, src, L, eo)
            assert true <= rsq * 1.05, (prec, eo, rsq, true, ra.final_iter)
            assert abs(ra.final_rsq - true) <= 0.05 * true + 1e-26
            assert ra.final_iter > 0 and ra.final_restart <= 1
            # same system solved by the FP64 oracle: solutions agree to the
            # accuracy the residual allows (condition number ~ 1/m^2)
            oia, ora = O.InvertArg(1e9, 20000, 20000, 5, eo), O.ResidArg(rsq, 0, 0, 0, 0, 0)
            ref, _ = fo.invert(m, src, oia, ora)
            assert rel_norm_err(half(got, L, eo), half(ref, L, eo)) <= max(1e-6, 30 * np.sqrt(rsq) / m ** 2)
            q.destroy_V(hin)
            q.destroy_V(hout)
    assert q.set_opts(prec_sloppy=64) == 0
    q.destroy_L(fla)


def test_mixed_iterations_close_to_fp64():
    """FP16 storage costs a bounded number of extra iterations."""
    L = (8, 8, 8, 8)
    q = gpu_lattice(L, "D")
    fat, lng = asqtad_links(L, 0.3, 7)
    fla = q.create_L_from_raw(fat, lng)
    src = LT.gaussian_vector(L, 102)
    its = {}
    for prec in (64, 32, 16):
        q.set_opts(prec_sloppy=prec)
        ia = QOP_invert_arg_t(1e9, 20000, 20000, 5, 0)
        ra = QOP_resid_arg_t(1e-20, 0, 0, 0, 0, 0)
        hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
        q.invert(fla, 0.02, hout, hin, ia, ra)
        its[prec] = ra.final_iter
        assert ra.final_rsq <= 1.05e-20
        q.destroy_V(hin)
        q.destroy_V(hout)
    q.set_opts(prec_sloppy=64)
    assert its[32] <= 1.3 * its[64] + 20 and its[16] <= 2.0 * its[64] + 50, its
    q.destroy_L(fla)
