"""Decomposed lattice on one GPU: directions marked with QOPB_dd_self_split
are treated as split between processes with this process as its own
neighbour, so every hop along them reads halos (packed, exchanged and
consumed exactly as between two GPUs) and the reductions take the decomposed
path.  The results must equal the single-domain results on the same inputs
and the oracle.  The exchange runs once through device copies (no
communicator) and once through a one-process NCCL communicator (NCCL sends
to and receives from itself).  Reference: QOP_init with a machine size and
QDP's halo exchange (lib/common.c:40-83, lib/layout_user.c:79-258)."""
import itertools

import numpy as np
import pytest

import conftest
import oracle as O
from conftest import gpu_lattice
from helpers import asqtad_links, eo_residual, full_residual, half, rel_norm_err, site_rel_err
from qopqdp_b200 import lattice as LT
from qopqdp_b200.qop import QOP_EVEN, QOP_EVENODD, QOP_ODD, QOP_invert_arg_t, QOP_resid_arg_t, Qop

pytestmark = pytest.mark.gpu

L = (4, 6, 4, 8)
V = int(np.prod(L))
COMBOS = list(itertools.product([0, 1, 2], [0, 1, 2]))


def run_suite(q, prec):
    """Every decomposition-aware entry point on fixed inputs; returns arrays."""
    dt = q.dtype
    assert q.set_opts(prec_sloppy=64, cg=0) == 0   # the reference algorithm in both runs
    fat, lng = asqtad_links(L, 0.4, 11)
    fla = q.create_L_from_raw([a.astype(dt) for a in fat], [a.astype(dt) for a in lng])
    src = LT.gaussian_vector(L, 31).astype(dt)
    init = LT.gaussian_vector(L, 32).astype(dt)
    res = {}

    def vec(a):
        return q.create_V(a)

    for eo_out, eo_in in COMBOS:
        hin, hout = vec(src), vec(init)
        q.dslash(fla, 0.0173, hout, hin, eo_out, eo_in)
        res["dslash", eo_out, eo_in] = q.extract_V(hout, V)
        q.destroy_V(hin)
        q.destroy_V(hout)
    for mu, fb in itertools.product(range(4), (1, -1)):
        hin, hout = vec(src), vec(init)
        q.dslash_dir(fla, mu, fb, 0.7, -1.3, hout, hin, QOP_EVENODD)
        res["dir", mu, fb] = q.extract_V(hout, V)
        q.destroy_V(hin)
        q.destroy_V(hout)
    for eo in (QOP_EVEN, QOP_ODD):
        hin, hout = vec(src), vec(init)
        n2 = q.ddagd_norm2(fla, 0.05, hout, hin, eo)
        res["ddagd", eo] = q.extract_V(hout, V)
        res["norm2", eo] = np.array([n2])
        q.destroy_V(hin)
        q.destroy_V(hout)
    rsq = 1e-16 if prec == "D" else 1e-10
    for eo in (QOP_EVENODD, QOP_EVEN):
        hin, hout = vec(src), vec(np.zeros_like(src))
        ra = QOP_resid_arg_t(rsq, 0, 0, 0, 0, 0)
        info = q.invert(fla, 0.03, hout, hin, QOP_invert_arg_t(1e9, 3000, 3000, 5, eo), ra)
        assert info.status == 0
        res["invert", eo] = q.extract_V(hout, V)
        res["iters", eo] = np.array([ra.final_iter])
        q.destroy_V(hin)
        q.destroy_V(hout)
    masses = [0.03, 0.11]
    hin = vec(src)
    outs = [vec(np.zeros_like(src)) for _ in masses]
    ras = [QOP_resid_arg_t(rsq, 0, 0, 0, 0, 0) for _ in masses]
    info = q.invert_multi(fla, [masses], [outs], [hin], QOP_invert_arg_t(1e9, 3000, 3000, 5, QOP_EVEN), [ras])
    assert info.status == 0
    for j, h in enumerate(outs):
        res["multi", j] = q.extract_V(h, V)
        q.destroy_V(h)
    q.destroy_V(hin)
    q.destroy_L(fla)
    return res, fat, lng, src, init


def reinit(q, mask, comm):
    if q.lib.QOP_is_initialized():
        q.finalize()
    conftest._state["L"] = None
    q.comm_finalize()
    if comm:
        uid = q.comm_unique_id()
        assert q.comm_init(uid, 1, 0) == 0
    assert q.dd_self_split(mask) == 0
    assert q.init(L) == 0


def restore(q):
    if q.lib.QOP_is_initialized():
        q.finalize()
    q.dd_self_split(0)
    q.comm_finalize()
    conftest._state["L"] = None


@pytest.mark.parametrize("prec,mask,comm", [("D", 15, False), ("F", 15, False), ("D", 5, True), ("F", 10, True)])
def test_self_split_matches_single_domain(prec, mask, comm):
    q = gpu_lattice(L, prec)
    base, fat, lng, src, init = run_suite(q, prec)
    try:
        reinit(q, mask, comm)
        info = q.dd_info()
        assert info["rank"] == 0 and info["mask"] == mask and info["local"] == L
        assert q.lib.QOP_sites_on_node_raw_V(QOP_EVENODD) == V
        split, *_ = run_suite(q, prec)
        tol = 1e-13 if prec == "D" else 2e-6
        for key, want in base.items():
            got = split[key]
            if key[0] in ("dslash", "dir", "ddagd"):
                assert site_rel_err(got, want) <= tol, key
            elif key[0] == "norm2":
                assert abs(got[0] - want[0]) <= tol * abs(want[0]), key
            elif key[0] == "iters":
                # the halo terms are summed in another order: CG at a 1e-16
                # target amplifies that rounding into a few % of iterations
                assert abs(int(got[0]) - int(want[0])) <= 0.05 * want[0] + 3, (key, got, want)
            else:   # solutions of the same system to the same target
                assert rel_norm_err(got, want) <= (1e-7 if prec == "D" else 1e-3), key
        # and against the oracle
        fo = O.Fla(O.Lattice(L), fat, lng)
        for eo_out, eo_in in COMBOS:
            ref = fo.dslash(float(q.real(0.0173).value), src.astype(np.float64), eo_out, eo_in,
                            out=init.astype(np.float64))
            assert site_rel_err(split["dslash", eo_out, eo_in], ref) <= tol
        true = full_residual(fo, float(q.real(0.03).value), split["invert", QOP_EVENODD].astype(np.float64),
                             src.astype(np.float64))
        assert true <= (1.05e-16 if prec == "D" else 5e-8)
    finally:
        restore(q)


def test_decomposed_lattice_refuses_single_domain_entry_points():
    q = Qop("D")
    try:
        reinit(q, 3, False)
        G = q.create_G([LT.random_gauge(L, 0.3, 5)[mu] for mu in range(4)])
        with pytest.raises(RuntimeError, match="status 1"):   # QOP_FAIL: staples cross the block faces
            q.create_L_from_G((1, 0.1, 0.1, 0.1, 0.1, 0.1), G)
        assert q.lib.QOPB_lattice_create((q.lib.QOPB_lattice_create.argtypes[0]._type_ * 4)(*L)) == -1
        assert q.lib.QOPB_serve_start() == -1
        q.destroy_G(G)
    finally:
        restore(q)


class _KStat(__import__("ctypes").Structure):
    _fields_ = [("name", __import__("ctypes").c_char * 32), ("launches", __import__("ctypes").c_int),
                ("total_ms", __import__("ctypes").c_double), ("bytes_per_launch", __import__("ctypes").c_double)]


def _prof_classes(q):
    import ctypes as C
    q.lib.QOPB_prof_end.argtypes = [C.POINTER(_KStat), C.c_int]
    buf = (_KStat * 32)()
    n = q.lib.QOPB_prof_end(buf, 32)
    return {buf[i].name.decode(): buf[i].launches for i in range(min(n, 32))}


@pytest.mark.parametrize("mask,comm", [(15, False), (9, True)])
def test_int16_mixed_solver_on_decomposed_lattice(mask, comm):
    """The int16 reliable-update solver (fused iteration, packed hop) on a
    decomposed lattice: int16 halo records, down-halo products formed with
    the FP64 links, and the step scalars computed after the all-reduce.  Each
    solve reaches the FP64 target with the iteration count and solution of
    the same solve on the undecomposed lattice, and runs the decomposed int16
    kernels (not an FP64 fallback)."""
    q = gpu_lattice(L, "D")
    fat, lng = asqtad_links(L, 0.4, 11)
    fo = O.Fla(O.Lattice(L), fat, lng)

    def solves():
        fla = q.create_L_from_raw(fat, lng)
        assert q.set_opts(prec_sloppy=16, cg=0) == 0
        out = {}
        q.lib.QOPB_prof_begin()
        for eo, m, seed in ((QOP_EVEN, 0.03, 41), (QOP_ODD, 0.01, 42)):
            src = LT.gaussian_vector(L, seed)
            hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
            ra = QOP_resid_arg_t(1e-20, 0, 0, 0, 0, 0)
            info = q.invert(fla, m, hout, hin, QOP_invert_arg_t(1e9, 20000, 20000, 5, eo), ra)
            assert info.status == 0
            out[eo] = (q.extract_V(hout, V), ra.final_iter, src, m)
            q.destroy_V(hin)
            q.destroy_V(hout)
        out["prof"] = _prof_classes(q)
        assert q.set_opts(prec_sloppy=64) == 0
        q.destroy_L(fla)
        return out

    base = solves()
    try:
        reinit(q, mask, comm)
        split = solves()
        assert split["prof"].get("hop_q16_upd_linkq16", 0) > 0, split["prof"]
        for eo in (QOP_EVEN, QOP_ODD):
            got, it, src, m = split[eo]
            want, it0, _, _ = base[eo]
            assert eo_residual(fo, m, got, src, L, eo) <= 1.05e-20, eo
            assert abs(it - it0) <= 0.05 * it0 + 3, (eo, it, it0)
            assert rel_norm_err(half(got, L, eo), half(want, L, eo)) <= 1e-8, eo
    finally:
        restore(q)


def test_eigcg_on_decomposed_lattice():
    """eigCG (option cg = 1) on a lattice decomposed in all four directions:
    its operator applications read halos and its inner products are summed
    over the decomposition, so it accumulates the same low modes as on the
    undecomposed lattice."""
    q = gpu_lattice(L, "D")
    fat, lng = asqtad_links(L, 0.4, 11)
    fo = O.Fla(O.Lattice(L), fat, lng)

    def run():
        fla = q.create_L_from_raw(fat, lng)
        assert q.set_opts(prec_sloppy=64, cg=1, eigcg_nev=6, eigcg_m=30, eigcg_l=120) == 0
        its = []
        for s in range(4):
            src = LT.gaussian_vector(L, 500 + s)
            src[V // 2:] = 0
            hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
            ra = QOP_resid_arg_t(1e-16, 0, 0, 0, 0, 0)
            assert q.invert(fla, 0.02, hout, hin, QOP_invert_arg_t(1e9, 5000, 5000, 5, QOP_EVENODD), ra).status == 0
            got = q.extract_V(hout, V)
            assert full_residual(fo, 0.02, got, src) <= 1.05e-16
            its.append(ra.final_iter)
            q.destroy_V(hin)
            q.destroy_V(hout)
        lam = q.eigcg_values(fla, QOP_EVEN)
        assert q.set_opts(cg=0) == 0
        q.destroy_L(fla)
        return its, lam

    its0, lam0 = run()
    try:
        reinit(q, 15, False)
        its1, lam1 = run()
        assert len(lam1) == len(lam0)
        assert np.allclose(lam1[:4], lam0[:4], rtol=1e-6, atol=0), (lam0[:4], lam1[:4])
        assert all(abs(a - b) <= 0.05 * b + 3 for a, b in zip(its1, its0)), (its0, its1)
    finally:
        restore(q)


def test_decomposed_lattice_without_naik_links():
    """Links without the Naik term (8 slots: halo depth 1, one product slab)
    on a lattice decomposed in all four directions: the nine Dslash cases
    match the oracle, and FP64 and int16 solves reach their targets with the
    iteration counts of the undecomposed lattice."""
    q = gpu_lattice(L, "D")
    fat, _ = asqtad_links(L, 0.4, 12, naik=False)
    fo = O.Fla(O.Lattice(L), fat, None)
    src = LT.gaussian_vector(L, 61)
    init = LT.gaussian_vector(L, 62)

    def run():
        fla = q.create_L_from_raw(fat, None)
        out = {}
        for eo_out, eo_in in COMBOS:
            hin, hout = q.create_V(src), q.create_V(init)
            q.dslash(fla, 0.05, hout, hin, eo_out, eo_in)
            out[eo_out, eo_in] = q.extract_V(hout, V)
            q.destroy_V(hin)
            q.destroy_V(hout)
        for prec in (64, 16):
            assert q.set_opts(prec_sloppy=prec, cg=0) == 0
            hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
            ra = QOP_resid_arg_t(1e-20, 0, 0, 0, 0, 0)
            assert q.invert(fla, 0.05, hout, hin, QOP_invert_arg_t(1e9, 20000, 20000, 5, QOP_EVEN), ra).status == 0
            got = q.extract_V(hout, V)
            assert eo_residual(fo, 0.05, got, src, L, QOP_EVEN) <= 1.05e-20, prec
            out["its", prec] = ra.final_iter
            q.destroy_V(hin)
            q.destroy_V(hout)
        assert q.set_opts(prec_sloppy=64) == 0
        q.destroy_L(fla)
        return out

    base = run()
    try:
        reinit(q, 15, True)
        split = run()
        for eo_out, eo_in in COMBOS:
            ref = fo.dslash(0.05, src, eo_out, eo_in, out=init.copy())
            assert site_rel_err(split[eo_out, eo_in], ref) <= 1e-13, (eo_out, eo_in)
        for prec in (64, 16):
            a, b = split["its", prec], base["its", prec]
            assert abs(a - b) <= 0.05 * b + 3, (prec, a, b)
    finally:
        restore(q)
