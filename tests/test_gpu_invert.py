"""Inverter parity through the C ABI (lib/asqtad_invert_p.c): EVEN / ODD
sources (solve_multi + refine + CGMS), EVENODD sources (project, CG,
reconstruct), invert_multi (flattened multi-mass, EVENODD two-source trick
and per-source CGMS), mixed_rsq restarts, relmin stopping, zero sources and
iteration exhaustion.  Each solve's true residual is checked in FP64 with the
oracle's operator (examples/asqtad_test.c:84-130), and solutions are compared
with the oracle's solve of the same system."""
import numpy as np
import pytest

import oracle as O
from conftest import gpu_lattice
from helpers import asqtad_links, hisq_links, eo_residual, full_residual, rel_norm_err, half
from qopqdp_b200 import lattice as LT
from qopqdp_b200.qop import QOP_invert_arg_t, QOP_resid_arg_t

pytestmark = pytest.mark.gpu

L = (4, 4, 4, 8)
V = int(np.prod(L))


def links(prec, kind="asqtad"):
    q = gpu_lattice(L, prec)
    if kind == "asqtad":
        fat, lng = asqtad_links(L, 0.3, 7)
    else:
        fat, lng, _, _ = hisq_links(L, 0.5, 9)
    dt = q.dtype
    fat = [np.asarray(a, dtype=dt) for a in fat]
    lng = [np.asarray(a, dtype=dt) for a in lng]
    fo = O.Fla(O.Lattice(L), [a.astype(np.float64) for a in fat], [a.astype(np.float64) for a in lng])
    return q, q.create_L_from_raw(fat, lng), fo


def args(evenodd, rsqmin, max_iter=2000, restart=1000, max_restarts=5, mixed=1e9, relmin=0.0):
    ia = QOP_invert_arg_t(mixed, max_iter, restart, max_restarts, evenodd)
    ra = QOP_resid_arg_t(rsqmin, 0, relmin, 0, 0, 0)
    return ia, ra


@pytest.mark.parametrize("prec,rsq", [("D", 1e-20), ("F", 1e-10)])
@pytest.mark.parametrize("eo", [0, 1])
def test_invert_eo_source(prec, rsq, eo):
    q, fla, fo = links(prec)
    m = 0.1
    src = LT.gaussian_vector(L, 40 + eo).astype(q.dtype)
    ia, ra = args(eo, rsq)
    hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
    info = q.invert(fla, m, hout, hin, ia, ra)
    assert info.status == 0
    got = q.extract_V(hout, V)
    # reference conventions: out = m A^{-1} in on the subset
    true = eo_residual(fo, float(q.real(m).value), got.astype(np.float64), src.astype(np.float64), L, eo)
    assert true <= rsq * (1.05 if prec == "D" else 50), true
    # F3 evaluates its final residual in single precision
    assert abs(ra.final_rsq - true) <= (0.05 if prec == "D" else 0.5) * true + (1e-24 if prec == "D" else 1e-12)
    assert (ia.max_iter, ra.rsqmin) == (2000, rsq)   # restored on return
    oia, ora = O.InvertArg(1e9, 2000, 1000, 5, eo), O.ResidArg(rsq, 0, 0, 0, 0, 0)
    ref, _ = fo.invert(float(q.real(m).value), src.astype(np.float64), oia, ora)
    assert rel_norm_err(half(got, L, eo), half(ref, L, eo)) <= (1e-8 if prec == "D" else 1e-4)
    if prec == "D":
        # FP64 rounding differs between the device reductions and the oracle's
        # OpenMP reductions (whose order depends on the host's thread count)
        assert abs(ra.final_iter - ora.final_iter) <= 0.02 * ora.final_iter + 3
    # examples/asqtad_test.c:101-127: re-solving from the solution needs
    # (almost) no iterations
    ia2, ra2 = args(eo, rsq)
    assert q.invert(fla, m, hout, hin, ia2, ra2).status == 0
    assert ra2.final_iter <= 2, ra2.final_iter
    q.destroy_V(hin)
    q.destroy_V(hout)
    q.destroy_L(fla)


@pytest.mark.parametrize("eo", [0, 1])
def test_mixed_solver_restart_from_solution(eo):
    """The int16 mixed solver started from a converged FP64 solution stops
    after its first true-residual check (asqtad_test.c:101-127)."""
    q, fla, fo = links("D")
    m = 0.05
    src = LT.gaussian_vector(L, 60 + eo)
    hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
    try:
        assert q.set_opts(prec_sloppy=16) == 0
        ia, ra = args(eo, 1e-20)
        assert q.invert(fla, m, hout, hin, ia, ra).status == 0
        first = ra.final_iter
        ia2, ra2 = args(eo, 1e-20)
        assert q.invert(fla, m, hout, hin, ia2, ra2).status == 0
        got = q.extract_V(hout, V)
        assert eo_residual(fo, m, got, src, L, eo) <= 1.05e-20
        assert ra2.final_iter <= 2, (first, ra2.final_iter)
    finally:
        q.set_opts(prec_sloppy=64)
        q.destroy_V(hin)
        q.destroy_V(hout)
        q.destroy_L(fla)


@pytest.mark.parametrize("prec,rsq", [("D", 1e-20), ("F", 1e-10)])
def test_invert_evenodd_source(prec, rsq):
    q, fla, fo = links(prec, "hisq")
    m = 0.05
    src = LT.gaussian_vector(L, 50).astype(q.dtype)
    ia, ra = args(2, rsq)
    hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
    q.invert(fla, m, hout, hin, ia, ra)
    got = q.extract_V(hout, V)
    true = full_residual(fo, float(q.real(m).value), got.astype(np.float64), src.astype(np.float64))
    assert true <= rsq * (1.05 if prec == "D" else 100), true
    assert abs(ra.final_rsq - true) <= 0.05 * true + 1e-24
    oia, ora = O.InvertArg(1e9, 2000, 1000, 5, 2), O.ResidArg(rsq, 0, 0, 0, 0, 0)
    ref, _ = fo.invert(float(q.real(m).value), src.astype(np.float64), oia, ora)
    assert rel_norm_err(got, ref) <= (1e-8 if prec == "D" else 1e-4)
    q.destroy_V(hin)
    q.destroy_V(hout)
    q.destroy_L(fla)


def _multi(q, fla, masses, srcs, ia, rsq):
    ras = [[QOP_resid_arg_t(rsq, 0, 0, 0, 0, 0) for _ in ms] for ms in masses]
    hins = [q.create_V(s) for s in srcs]
    houts = [[q.create_V(np.zeros_like(srcs[0])) for _ in ms] for ms in masses]
    info = q.invert_multi(fla, masses, houts, hins, ia, ras)
    outs = [[q.extract_V(h, V).astype(np.float64) for h in row] for row in houts]
    for h in hins:
        q.destroy_V(h)
    for row in houts:
        for h in row:
            q.destroy_V(h)
    return info, ras, outs


@pytest.mark.parametrize("prec", ["D", "F"])
def test_invert_multi_eo_single_source_converges(prec):
    """One source, several masses: solve_multi + CGMS reach every tolerance."""
    q, fla, fo = links(prec, "hisq")
    rsq = 1e-20 if prec == "D" else 1e-10
    masses = [[0.02, 0.05, 0.2]]
    srcs = [LT.gaussian_vector(L, 60).astype(q.dtype)]
    ia, _ = args(0, rsq, max_iter=8000, max_restarts=20)
    info, ras, outs = _multi(q, fla, masses, srcs, ia, rsq)
    assert info.status == 0
    for j, m in enumerate(masses[0]):
        true = eo_residual(fo, float(q.real(m).value), outs[0][j], srcs[0].astype(np.float64), L, 0)
        assert true <= rsq * (1.1 if prec == "D" else 100), (m, true)
    q.destroy_L(fla)


def test_invert_multi_eo_several_sources_matches_oracle():
    """Several sources flattened into one solve_multi (asqtad_invert_p.c:893-912).
    The reference's refine indexes m2 by the unique-mass index (:300), so solves
    whose mass order differs from the sorted mass list stall; the device path
    reproduces the reference result rather than converging."""
    q, fla, fo = links("D", "hisq")
    rsq = 1e-20
    masses = [[0.02, 0.05, 0.2], [0.1]]
    srcs = [LT.gaussian_vector(L, 60 + s) for s in range(2)]
    ia, _ = args(0, rsq, max_iter=8000, max_restarts=20)
    info, ras, outs = _multi(q, fla, masses, srcs, ia, rsq)
    oras = [[O.ResidArg(rsq, 0, 0, 0, 0, 0) for _ in ms] for ms in masses]
    fo.invert_multi(masses, srcs, O.InvertArg(1e9, 8000, 1000, 20, 0), oras)
    for s, ms in enumerate(masses):
        for j, m in enumerate(ms):
            g, o = ras[s][j].final_rsq, oras[s][j].final_rsq
            true = eo_residual(fo, m, outs[s][j], srcs[s], L, 0)
            assert abs(true - g) <= 0.05 * g + 1e-24                 # reported = true residual
            assert (g <= rsq * 1.1 and o <= rsq * 1.1) or 0.2 <= g / o <= 5, (s, m, g, o)
            assert abs(ras[s][j].final_iter - oras[s][j].final_iter) <= 0.02 * oras[s][j].final_iter + 3
    q.destroy_L(fla)


@pytest.mark.parametrize("masses", [[[0.05], [0.1]], [[0.05, 0.1, 0.3]]])
def test_invert_multi_evenodd_paths(masses):
    """EVENODD invert_multi: two-source trick or per-source CGMS on the even
    subset, then out *= m (asqtad_invert_p.c:937-1050).  CGMS stops on the
    shift with the largest rsqmin (ties: the last one), so lighter masses are
    returned unconverged exactly as the reference returns them."""
    q, fla, fo = links("D")
    rsq = 1e-16
    nsrc = len(masses)
    srcs = [LT.gaussian_vector(L, 70 + s) for s in range(nsrc)]
    ia, _ = args(2, rsq)
    info, ras, outs = _multi(q, fla, masses, srcs, ia, rsq)
    oras = [[O.ResidArg(rsq, 0, 0, 0, 0, 0) for _ in ms] for ms in masses]
    refs, _ = fo.invert_multi(masses, srcs, O.InvertArg(1e9, 2000, 1000, 5, 2), oras)
    for s, ms in enumerate(masses):
        for j, m in enumerate(ms):
            assert abs(ras[s][j].final_iter - oras[s][j].final_iter) <= 0.02 * oras[s][j].final_iter + 3
            g, o = ras[s][j].final_rsq, oras[s][j].final_rsq
            if o <= 1.05 * rsq:   # converged: the same residual
                assert abs(g - o) <= 0.1 * o + 1e-20, (s, m, g, o)
            else:   # returned unconverged: its residual moves a few per cent per
                # iteration, and the oracle's iteration count moves with its
                # OpenMP thread count (0.00486-0.0057 for m = 0.05 across hosts)
                assert 0.5 * o <= g <= 2 * o, (s, m, g, o)
            assert rel_norm_err(half(outs[s][j], L, 0), half(refs[s][j], L, 0)) <= 1e-3
    q.destroy_L(fla)


def test_mixed_rsq_restart_reaches_fp64_tolerance():
    """D3 with mixed_rsq: inner restarts run in FP32 (asqtad_invert_p.c:510-537)
    yet the FP64-refined result meets the requested squared residual."""
    q, fla, fo = links("D", "hisq")
    rsq = 1e-20
    src = LT.gaussian_vector(L, 80)
    ia, ra = args(0, rsq, mixed=1e-5, max_restarts=20)
    hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
    q.invert(fla, 0.05, hout, hin, ia, ra)
    got = q.extract_V(hout, V)
    assert eo_residual(fo, 0.05, got, src, L, 0) <= rsq * 1.1
    assert ra.final_restart >= 1
    q.destroy_V(hin)
    q.destroy_V(hout)
    q.destroy_L(fla)


def test_relmin_and_edge_cases():
    q, fla, fo = links("D")
    src = LT.gaussian_vector(L, 90)
    # Fermilab relative residual stopping (invert_utilities_p.c:1-40)
    ia, ra = args(2, 0.0, relmin=1e-14)
    hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
    q.invert(fla, 0.1, hout, hin, ia, ra)
    oia, ora = O.InvertArg(1e9, 2000, 1000, 5, 2), O.ResidArg(0.0, 0, 1e-14, 0, 0, 0)
    ref, _ = fo.invert(0.1, src, oia, ora)
    assert ra.final_rel <= 1e-14 * 1.01 and abs(ra.final_iter - ora.final_iter) <= 0.02 * ora.final_iter + 3
    # zero source: zero solution, zero residual
    z = np.zeros_like(src)
    hz, hzo = q.create_V(z), q.create_V(src)
    ia, ra = args(0, 1e-20)
    q.invert(fla, 0.1, hzo, hz, ia, ra)
    assert not q.extract_V(hzo, V)[: V // 2].any() and ra.final_rsq == 0
    # iteration exhaustion: stops at max_iter without converging
    ia, ra = args(0, 1e-30, max_iter=37, restart=1000, max_restarts=1)
    hout2 = q.create_V(np.zeros_like(src))
    q.invert(fla, 0.01, hout2, hin, ia, ra)
    assert ra.final_rsq > 1e-30 and ra.final_iter <= 37 + 4
    for h in (hin, hout, hz, hzo, hout2):
        q.destroy_V(h)
    q.destroy_L(fla)


def test_invalid_handles_report_fail():
    q = gpu_lattice(L, "D")
    from qopqdp_b200.qop import QOP_info_t
    info = QOP_info_t()
    q.dslash(None, 0.1, None, None, 2, 2, info=info)
    assert info.status == 1
    ia, ra = args(0, 1e-10)
    info = QOP_info_t()
    q.invert(None, 0.1, None, None, ia, ra, info=info)
    assert info.status == 1
