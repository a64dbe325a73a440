"""The device path against the reference's own outputs.

tests/golden/qopref_4x4x4x4.npz holds what the reference's unmodified
sources (compiled by oracle/ref) computed on seeded 4^4 inputs:
rephased gauge and link checksums, asqtad Dslash, an EVEN solve,
invert_multi on ODD and a HISQ Dslash (tests/golden/make_qopref_golden.py
lists them).  Here the whole chain runs on the GPU through the C ABI --
gauge upload, QOP_rephase_G, QOP_asqtad_create_L_from_G /
QOP_hisq_create_L_from_G, Dslash, invert (FP64 and the int16 mixed
solver), invert_multi -- and is compared with those outputs directly.
"""
import os

import numpy as np
import pytest

from conftest import gpu_lattice
from helpers import rel_norm_err
from qopqdp_b200 import lattice as LT
from qopqdp_b200.qop import QOP_invert_arg_t, QOP_resid_arg_t

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "qopref_4x4x4x4.npz")
L = (4, 4, 4, 4)
V = 256


def checksum(arrs):
    a = np.concatenate([np.asarray(x, dtype=np.float64).ravel() for x in arrs])
    w = np.cos(0.37 * np.arange(a.size))
    return np.array([float((a * a).sum()), float((a * w).sum())])


def close_ck(a, b, tol):
    return np.all(np.abs(np.asarray(a) - np.asarray(b)) <= tol * (1 + np.abs(np.asarray(b))))


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def _gauge(q, d):
    U = LT.random_gauge(L, 0.3, 7)
    assert close_ck(checksum(U), d["gauge_ck"], 1e-12), "gauge generator changed"
    hG = q.create_G([np.asarray(u, dtype=q.dtype) for u in U])
    q.rephase_G(hG, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
    return hG


@pytest.mark.parametrize("prec", ["D", "F"])
def test_device_links_and_dslash_match_reference(gold, prec):
    d = gold
    q = gpu_lattice(L, prec)
    tol_ck, tol = (1e-12, 1e-13) if prec == "D" else (1e-5, 2e-6)
    hG = _gauge(q, d)
    assert close_ck(checksum(q.extract_G(hG, V)), d["rephased_ck"], tol_ck)
    fla = q.create_L_from_G(LT.ASQTAD_BENCH_COEFFS, hG)
    fat, lng = q.extract_L(fla, V)
    assert close_ck(checksum(fat), d["asq_fat_ck"], tol_ck)
    assert close_ck(checksum(lng), d["asq_long_ck"], tol_ck)
    src = LT.gaussian_vector(L, 41).astype(q.dtype)
    hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
    for eo_out, eo_in, key in ((2, 2, "asq_dslash_eoeo"), (0, 1, "asq_dslash_e_o")):
        q.dslash(fla, 0.1, hout, hin, eo_out, eo_in)
        got = q.extract_V(hout, V).reshape(V, 6).astype(np.float64)
        ref = d[key]
        if eo_out == 0:
            got, ref = got[: V // 2], ref[: V // 2]
        assert rel_norm_err(got, ref) < tol, key
    q.destroy_L(fla)
    hh = q.hisq_create_L_from_G(LT.hisq_bench_coeffs(), hG)
    hfla = q.hisq_asqtad_links(hh)
    hfat, hlng = q.extract_L(hfla, V)
    assert close_ck(checksum(hfat), d["hisq_fat_ck"], 1e-11 if prec == "D" else 1e-5)
    assert close_ck(checksum(hlng), d["hisq_long_ck"], 1e-11 if prec == "D" else 1e-5)
    q.dslash(hfla, 0.05, hout, hin, 2, 2)
    got = q.extract_V(hout, V).reshape(V, 6).astype(np.float64)
    assert rel_norm_err(got, d["hisq_dslash_eoeo"]) < (1e-12 if prec == "D" else 2e-6)
    q.hisq_destroy_L(hh)
    q.destroy_V(hin)
    q.destroy_V(hout)
    q.destroy_G(hG)


@pytest.mark.parametrize("sloppy", [64, 16])
def test_device_solves_match_reference(gold, sloppy):
    """EVEN solve (the FP64 reference algorithm, and the int16 reliable-update
    solver that the benchmark times) and invert_multi on ODD: solutions
    agree with the reference's to 1e-8."""
    d = gold
    q = gpu_lattice(L, "D")
    hG = _gauge(q, d)
    fla = q.create_L_from_G(LT.ASQTAD_BENCH_COEFFS, hG)
    src = LT.gaussian_vector(L, 41)
    hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
    assert q.set_opts(prec_sloppy=sloppy) == 0
    try:
        ra = QOP_resid_arg_t(1e-20, 0, 0, 0, 0, 0)
        info = q.invert(fla, 0.1, hout, hin, QOP_invert_arg_t(1e9, 2000, 1000, 5, 0), ra)
        assert info.status == 0 and ra.final_rsq <= 1e-20
        got = q.extract_V(hout, V).reshape(V, 6)[: V // 2]
        assert rel_norm_err(got, d["asq_invert_even"]) < 1e-8
        if sloppy == 64:
            assert abs(ra.final_iter - int(d["asq_invert_even_iters"][0])) <= 0.02 * ra.final_iter + 3
        masses = [0.1, 0.2, 0.4]
        ras = [QOP_resid_arg_t(1e-20, 0, 0, 0, 0, 0) for _ in masses]
        houts = [q.create_V(np.zeros_like(src)) for _ in masses]
        info = q.invert_multi(fla, [masses], [houts], [hin], QOP_invert_arg_t(1e9, 2000, 1000, 5, 1), [ras])
        assert info.status == 0
        for k, h in enumerate(houts):
            got = q.extract_V(h, V).reshape(V, 6)[V // 2:]
            assert ras[k].final_rsq <= 1e-20
            assert rel_norm_err(got, d["asq_multi_odd"][k]) < 1e-8, k
            q.destroy_V(h)
    finally:
        assert q.set_opts(prec_sloppy=64) == 0
    q.destroy_V(hin)
    q.destroy_V(hout)
    q.destroy_L(fla)
    q.destroy_G(hG)


def test_device_forces_match_reference(gold):
    """Fermion forces on the device (FP64) against the reference's on a rough
    field with two filtered fat7 links: the asqtad force by ASVEC (one
    source) and FNMAT (three), and the HISQ force with two Naik groups and
    the default force filter, whose W-level derivative carries the
    reference's Lepage term into the filtered U(3) adjoint."""
    d = gold
    q = gpu_lattice(L, "D")
    Ur = LT.random_gauge(L, 0.5, 2)
    assert close_ck(checksum(Ur), d["force_gauge_ck"], 1e-12), "gauge generator changed"
    hG = q.create_G([np.asarray(u, dtype=np.float64) for u in Ur])
    q.rephase_G(hG, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
    xs = [LT.gaussian_vector(L, 51 + i) for i in range(3)]
    hv = [q.create_V(x) for x in xs]
    eps = [0.3, -0.2, 0.5]
    zero = [np.zeros((V, 3, 3, 2)) for _ in range(4)]

    def agree(F, key, tol):
        got = np.stack([np.asarray(f, dtype=np.float64) for f in q.extract_F(F, V)]).reshape(d[key].shape)
        assert np.abs(got - d[key]).max() <= tol * np.abs(d[key]).max(), key

    for n, key in ((1, "force_asq_asvec"), (3, "force_asq_fnmat")):
        F = q.create_F(zero)
        assert q.asqtad_force(hG, F, LT.ASQTAD_BENCH_COEFFS, eps[:n], hv[:n]).status == 0
        agree(F, key, 1e-12)
        q.destroy_F(F)
    hc = LT.hisq_bench_coeffs()
    hc.n_naiks = 2
    hc.eps_naik[1] = 0.1
    hc.difference_one_link, hc.difference_naik = 0.3, -0.05
    q.set_hisq_opts(want_aux=1)
    H = q.hisq_create_L_from_G(hc, hG)
    F = q.create_F(zero)
    assert q.hisq_force(H, F, hc, eps, hv, [2, 1]).status == 0
    agree(F, "force_hisq", 1e-9)
    q.destroy_F(F)
    q.hisq_destroy_L(H)
    for h in hv:
        q.destroy_V(h)
    q.destroy_G(hG)
