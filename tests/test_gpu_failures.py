"""Failure paths that the reference ends with exit() or leaves unchecked,
reported here through info->status and tested without faulting a GPU
(every failure is made on the host or by a wait that runs out):

* a NaN or Inf source: QOP_FAIL before any iteration (the reference would
  iterate on NaN; it aborts only on NaN inside u3_un_analytic,
  lib/hisq_reunit_utilities_p.c:172-184);
* a failed device allocation (injected on the host): QOP_MEM_ERROR from
  every allocation point of the solve paths, with nothing leaked
  (the reference's QOP_malloc calls exit(1), include/qop_internal.h:98-103);
* the solve service: an HBM budget that holds one engine makes a request on a
  second lattice wait for the first engine and then complete; a request with
  a NaN source fails alone;
* the bounded mbarrier waits of the TMA-staged int16 hop: a limit of zero
  polls runs out, the solve returns QOP_FAIL, the copies in flight are drained
  under the normal limit and the library keeps working.
"""
import numpy as np
import pytest

import oracle as O
from conftest import gpu_lattice
from devmem import Memory
from helpers import asqtad_links, eo_residual, hisq_links
from qopqdp_b200 import lattice as LT
from qopqdp_b200.qop import QOP_invert_arg_t, QOP_resid_arg_t

pytestmark = pytest.mark.gpu

QOP_SUCCESS, QOP_FAIL, QOP_MEM_ERROR = 0, 1, 3   # include/qop.h (reference qop_int.h:15-21)
L8 = (8, 8, 8, 8)


def _solve(q, fla, mass, hout, hin, eo, rsq=1e-20, inject=0):
    """one invert from a zero guess; inject = n makes its n-th device allocation fail"""
    q.dslash(fla, 0.0, hout, hout, 2, 2)                    # zero guess
    ia = QOP_invert_arg_t(1e9, 20000, 20000, 5, eo)
    ra = QOP_resid_arg_t(rsq, 0, 0, 0, 0, 0)
    assert q.lib.QOPB_inject_alloc_failure(inject) == 0
    info = q.invert(fla, mass, hout, hin, ia, ra)
    assert q.lib.QOPB_inject_alloc_failure(0) == 0
    return info.status, ra


def _multi(q, fla, masses, hin, hout, eo, inject=0):
    ia = QOP_invert_arg_t(1e9, 20000, 20000, 5, eo)
    ras = [[QOP_resid_arg_t(1e-20, 0, 0, 0, 0, 0) for _ in masses]]
    for h in hout:
        q.dslash(fla, 0.0, h, h, 2, 2)
    assert q.lib.QOPB_inject_alloc_failure(inject) == 0
    info = q.invert_multi(fla, [masses], [hout], [hin], ia, ras)
    assert q.lib.QOPB_inject_alloc_failure(0) == 0
    return info.status


@pytest.mark.parametrize("prec", ["D", "F"])
def test_nonfinite_source_fails(prec):
    q = gpu_lattice(L8, prec)
    fat, lng = asqtad_links(L8, 0.3, 7)
    dt = q.dtype
    fla = q.create_L_from_raw([np.asarray(a, dt) for a in fat], [np.asarray(a, dt) for a in lng])
    good = LT.gaussian_vector(L8, 900).astype(dt)
    hout = q.create_V(np.zeros_like(good))
    sloppy = (64, 16) if prec == "D" else (64,)
    for bad_value in (np.nan, np.inf):
        bad = good.copy()
        bad[17, 1, 0] = bad_value                               # an even site
        hbad = q.create_V(bad)
        for sp in sloppy:
            assert q.set_opts(prec_sloppy=sp) == 0
            for eo in (0, 2):
                st, _ = _solve(q, fla, 0.1, hout, hbad, eo)
                assert st == QOP_FAIL, (bad_value, sp, eo)
            assert _multi(q, fla, [0.1, 0.2], hbad, [q.create_V(np.zeros_like(good)) for _ in range(2)], 0) == QOP_FAIL
        q.destroy_V(hbad)
    # the library keeps working
    hgood = q.create_V(good)
    target = 1e-20 if prec == "D" else 1e-10
    for sp in sloppy:
        assert q.set_opts(prec_sloppy=sp) == 0
        st, ra = _solve(q, fla, 0.1, hout, hgood, 0, rsq=target)
        assert st == QOP_SUCCESS and ra.final_rsq <= target * 1.05
    assert q.set_opts(prec_sloppy=64) == 0
    q.destroy_V(hgood)
    q.destroy_V(hout)
    q.destroy_L(fla)


@pytest.mark.parametrize("path", ["invert_fp64", "invert_int16", "multi_int16", "evenodd_fp64"])
def test_allocation_failure_is_mem_error_and_leaks_nothing(path):
    q = gpu_lattice(L8, "D")
    fat, lng = asqtad_links(L8, 0.3, 7)
    fla = q.create_L_from_raw(fat, lng)
    src = LT.gaussian_vector(L8, 901)
    hin = q.create_V(src)
    hout = [q.create_V(np.zeros_like(src)) for _ in range(3)]
    sp = 16 if "int16" in path else 64
    assert q.set_opts(prec_sloppy=sp) == 0

    def call(n=0):
        if path == "multi_int16":
            return _multi(q, fla, [0.1, 0.15, 0.3], hin, hout, 0, inject=n)
        return _solve(q, fla, 0.1, hout[0], hin, 2 if path == "evenodd_fp64" else 0, inject=n)[0]

    assert call() == QOP_SUCCESS            # builds the cached link copies
    mem = Memory()
    base = mem.used()
    failures = 0
    for n in range(1, 200):
        st = call(n)
        if st == QOP_SUCCESS:
            break                           # the call makes fewer than n allocations
        assert st == QOP_MEM_ERROR, (path, n, st)
        failures += 1
        assert mem.used() == base, (path, n, mem.used() - base)
    else:
        raise AssertionError("the call never completed")
    assert failures >= 2, failures
    assert call() == QOP_SUCCESS
    assert mem.used() == base
    assert q.set_opts(prec_sloppy=64) == 0
    for h in [hin] + hout:
        q.destroy_V(h)
    q.destroy_L(fla)


def test_serve_hbm_budget_makes_a_second_lattice_wait():
    LA, LB = (4, 4, 4, 8), (8, 8, 8, 8)
    q = gpu_lattice(LA, "D")
    lb = q.lattice_create(LB)
    fa, la_, _, _ = hisq_links(LA, 0.5, 9)
    fb, lb_ = asqtad_links(LB, 0.3, 7)
    foa, fob = O.Fla(O.Lattice(LA), fa, la_), O.Fla(O.Lattice(LB), fb, lb_)
    assert q.lattice_use(0) == 0
    ha = q.create_L_from_raw(fa, la_)
    assert q.lattice_use(lb) == 0
    hb = q.create_L_from_raw(fb, lb_)
    assert q.lattice_use(0) == 0
    assert q.set_opts(serve_hbm_mb=-1) != 0
    assert q.set_opts(serve_hbm_mb=1) == 0          # room for one engine at a time
    a_src, c_src = LT.gaussian_vector(LB, 920), LT.gaussian_vector(LA, 921)
    a_dst, c_dst = [np.zeros_like(a_src)], [np.zeros_like(c_src)]
    nan_src = LT.gaussian_vector(LB, 922)
    nan_src[3, 0, 1] = np.nan
    nan_dst = [np.zeros_like(nan_src)]
    assert q.serve_start() == 0
    try:
        ta = q.serve_submit(hb, lb, 0, 0.005, 1e-20, [a_src], a_dst)    # long: m = 0.005 on 8^4
        assert q.serve_wait(ta, 0.05)[0] == 1
        tc = q.serve_submit(ha, 0, 1, 0.1, 1e-20, [c_src], c_dst)
        tn = q.serve_submit(hb, lb, 0, 0.1, 1e-20, [nan_src], nan_dst)      # joins A's engine
        rc_n, res_n = q.serve_wait(tn, 120.0)
        rc_c, res_c = q.serve_wait(tc, 120.0)
        rc_a, res_a = q.serve_wait(ta, 300.0)
    finally:
        assert q.serve_stop() == 0
        assert q.set_opts(serve_hbm_mb=0) == 0
    assert rc_a == rc_c == rc_n == 0
    assert res_n.status == QOP_FAIL                  # the NaN request fails alone
    assert res_a.status == res_c.status == QOP_SUCCESS
    # C waited for A's engine to be freed, then ran alone
    assert res_c.queue_ms >= 0.5 * res_a.solve_ms, (res_c.queue_ms, res_a.solve_ms)
    assert res_c.batch_systems == 1
    assert eo_residual(fob, 0.005, a_dst[0], a_src, LB, 0) <= 1e-20 * 1.05
    assert eo_residual(foa, 0.1, c_dst[0], c_src, LA, 1) <= 1e-20 * 1.05
    assert q.lattice_use(lb) == 0
    q.destroy_L(hb)
    assert q.lattice_use(0) == 0
    q.destroy_L(ha)


def test_tma_hop_wait_limit_runs_out_and_the_library_recovers():
    q = gpu_lattice(L8, "D")
    fat, lng = asqtad_links(L8, 0.3, 7)
    fo = O.Fla(O.Lattice(L8), fat, lng)
    fla = q.create_L_from_raw(fat, lng)
    src = LT.gaussian_vector(L8, 930)
    hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
    assert q.set_opts(mbar_tries=-1) != 0
    for variant in (1, 2):                           # the two TMA-staged int16 hops
        assert q.set_opts(prec_sloppy=16, hop_kernel=variant, mbar_tries=0) == 0   # every wait gives up at once
        st, _ = _solve(q, fla, 0.1, hout, hin, 0)
        assert st == QOP_FAIL, variant
        assert q.set_opts(mbar_tries=1 << 22) == 0
        st, ra = _solve(q, fla, 0.1, hout, hin, 0)
        assert st == QOP_SUCCESS, variant
        assert eo_residual(fo, 0.1, q.extract_V(hout, int(np.prod(L8))), src, L8, 0) <= 1e-20 * 1.05
    assert q.set_opts(prec_sloppy=64, hop_kernel=25) == 0
    q.destroy_V(hin)
    q.destroy_V(hout)
    q.destroy_L(fla)
