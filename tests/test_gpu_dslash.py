"""Dslash parity through the C ABI: every (eo_out, eo_in) combination of
QOP_D3/F3_asqtad_dslash (lib/asqtad_dslash_p.c:1048-1092), dslash_dir,
ddagd, ddagd_norm2 and diaginv against the FP64 oracle on identical inputs.
Tolerances: D3 <= 1e-13 and F3 <= 2e-6, relative, per site."""
import itertools

import numpy as np
import pytest

import oracle as O
from conftest import gpu_lattice
from helpers import asqtad_links, site_rel_err, hisq_links
from qopqdp_b200 import lattice as LT

pytestmark = pytest.mark.gpu

TOL = {"D": 1e-13, "F": 2e-6}
COMBOS = list(itertools.product([0, 1, 2], [0, 1, 2]))


def setup(L, prec, naik=True, kind="asqtad"):
    q = gpu_lattice(L, prec)
    if kind == "asqtad":
        fat, lng = asqtad_links(L, 0.3, 7, naik)
    else:
        fat, lng, _, _ = hisq_links(L, 0.5, 9)
    dt = np.float32 if prec == "F" else np.float64
    fat = [np.asarray(a, dtype=dt) for a in fat]
    lng = [np.asarray(a, dtype=dt) for a in lng] if lng is not None else None
    lat = O.Lattice(L)
    fo = O.Fla(lat, [a.astype(np.float64) for a in fat], [a.astype(np.float64) for a in lng] if lng else None)
    fla = q.create_L_from_raw(fat, lng)
    return q, fla, fo


@pytest.mark.parametrize("prec", ["D", "F"])
@pytest.mark.parametrize("L", [(4, 4, 4, 4), (4, 6, 4, 8)])
def test_dslash_all_eo_combos(prec, L):
    q, fla, fo = setup(L, prec)
    V = int(np.prod(L))
    src = LT.gaussian_vector(L, 3).astype(q.dtype)
    for mass in (0.1, 0.0173):
        for eo_out, eo_in in COMBOS:
            init = LT.gaussian_vector(L, 4).astype(q.dtype)
            hin = q.create_V(src)
            hout = q.create_V(init)
            q.dslash(fla, mass, hout, hin, eo_out, eo_in)
            got = q.extract_V(hout, V)
            ref = fo.dslash(float(q.real(mass).value), src.astype(np.float64), eo_out, eo_in,
                            out=init.astype(np.float64))
            err = site_rel_err(got, ref)
            assert err <= TOL[prec], (prec, L, mass, eo_out, eo_in, err)
            q.destroy_V(hin)
            q.destroy_V(hout)
    q.destroy_L(fla)


@pytest.mark.parametrize("prec", ["D", "F"])
def test_dslash_hisq_links_and_no_naik(prec):
    L = (4, 4, 4, 8)
    V = int(np.prod(L))
    for kind, naik in (("hisq", True), ("asqtad", False)):
        q, fla, fo = setup(L, prec, naik=naik, kind=kind)
        src = LT.gaussian_vector(L, 8).astype(q.dtype)
        hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
        q.dslash(fla, 0.05, hout, hin, 2, 2)
        ref = fo.dslash(float(q.real(0.05).value), src.astype(np.float64), 2, 2)
        assert site_rel_err(q.extract_V(hout, V), ref) <= TOL[prec]
        for h in (hin, hout):
            q.destroy_V(h)
        q.destroy_L(fla)


@pytest.mark.parametrize("prec", ["D", "F"])
def test_dslash_aliased_out_in(prec):
    """out == in: the reference hops from a temp copy, then applies the mass
    term to the overwritten field (asqtad_dslash_p.c:997-1092)."""
    L = (4, 4, 4, 4)
    q, fla, fo = setup(L, prec)
    V = int(np.prod(L))
    src = LT.gaussian_vector(L, 12).astype(q.dtype)
    for eo_out, eo_in in COMBOS:
        h = q.create_V(src)
        q.dslash(fla, 0.2, h, h, eo_out, eo_in)
        x = src.astype(np.float64).copy()
        O.lib().or_dslash(fo.h, float(q.real(0.2).value), O._p(x), O._p(x), eo_out, eo_in)
        assert site_rel_err(q.extract_V(h, V), x) <= TOL[prec], (eo_out, eo_in)
        q.destroy_V(h)
    q.destroy_L(fla)


@pytest.mark.parametrize("prec", ["D", "F"])
def test_ddagd_norm2_and_diaginv(prec):
    L = (4, 4, 4, 8)
    q, fla, fo = setup(L, prec)
    V = int(np.prod(L))
    src = LT.gaussian_vector(L, 21).astype(q.dtype)
    m = 0.07
    mm = float(q.real(m).value)
    for eo in (0, 1):
        hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
        n2 = q.ddagd_norm2(fla, m, hout, hin, eo)
        ref, rn2 = fo.ddagd_norm2(mm, src.astype(np.float64), eo)
        sl = slice(0, V // 2) if eo == 0 else slice(V // 2, V)
        assert site_rel_err(q.extract_V(hout, V)[sl], ref[sl]) <= TOL[prec] * 10
        assert abs(n2 - rn2) / rn2 <= TOL[prec] * 10
        q.ddagd(fla, m, hout, hin, eo)
        assert site_rel_err(q.extract_V(hout, V)[sl], ref[sl]) <= TOL[prec] * 10
        q.diaginv(fla, m, hout, hin, eo)
        assert site_rel_err(q.extract_V(hout, V)[sl], src[sl].astype(np.float64) / mm) <= TOL[prec]
        q.destroy_V(hin)
        q.destroy_V(hout)
    q.destroy_L(fla)


@pytest.mark.parametrize("prec", ["D", "F"])
def test_dslash_dir_accumulates(prec):
    L = (4, 4, 4, 4)
    q, fla, fo = setup(L, prec)
    V = int(np.prod(L))
    src = LT.gaussian_vector(L, 31).astype(q.dtype)
    base = LT.gaussian_vector(L, 32).astype(q.dtype)
    for mu, fb, eo in ((0, 1, 2), (3, -1, 0), (2, 1, 1)):
        hin, hout = q.create_V(src), q.create_V(base)
        q.dslash_dir(fla, mu, fb, 0.7, -1.3, hout, hin, eo)
        ref = fo.dslash_dir(mu, fb, 0.7, -1.3, src.astype(np.float64), eo, base.astype(np.float64).copy())
        assert site_rel_err(q.extract_V(hout, V), ref) <= TOL[prec] * 10
        q.destroy_V(hin)
        q.destroy_V(hout)
    q.destroy_L(fla)


def test_raw_roundtrip_keeps_other_parity():
    L = (4, 4, 4, 4)
    q = gpu_lattice(L, "D")
    V = int(np.prod(L))
    a = LT.gaussian_vector(L, 1)
    b = LT.gaussian_vector(L, 2)
    h = q.create_V(a, 0)                       # only the even half is read
    got = q.extract_V(h, V, 2)
    assert np.array_equal(got[: V // 2], a[: V // 2])
    assert not got[V // 2:].any()
    out = b.copy()
    q.extract_V(h, V, 1, into=out)             # only the odd half is written
    assert np.array_equal(out[: V // 2], b[: V // 2])
    q.destroy_V(h)


def test_profiler_samples_every_nth_launch():
    """QOPB_prof_every(n) brackets launches 0, n, 2n, ... of each kernel
    class with CUDA events (1, the default, brackets every launch; n < 1 is
    refused); the per-class counts follow, and every sampled class has a
    positive device time."""
    import ctypes as C

    class KStat(C.Structure):
        _fields_ = [("name", C.c_char * 32), ("launches", C.c_int), ("total_ms", C.c_double),
                    ("bytes_per_launch", C.c_double)]

    L = (4, 4, 4, 4)
    q, fla, _ = setup(L, "D")
    src = LT.gaussian_vector(L, 3)
    hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
    q.lib.QOPB_prof_end.argtypes = [C.POINTER(KStat), C.c_int]

    def classes(every, calls):
        assert q.lib.QOPB_prof_every(every) == 0
        q.lib.QOPB_prof_begin()
        for _ in range(calls):
            q.dslash(fla, 0.1, hout, hin, 1, 0)
        buf = (KStat * 32)()
        n = q.lib.QOPB_prof_end(buf, 32)
        return {buf[i].name.decode(): (buf[i].launches, buf[i].total_ms) for i in range(min(n, 32))}

    try:
        assert q.lib.QOPB_prof_every(0) == -1
        full, samp = classes(1, 10), classes(4, 10)
    finally:
        q.lib.QOPB_prof_every(1)
        q.destroy_V(hin)
        q.destroy_V(hout)
        q.destroy_L(fla)
    assert full and set(full) == set(samp)
    for name, (n, ms) in full.items():
        assert n >= 10 and n % 10 == 0 and ms > 0, (name, n, ms)
        assert samp[name][0] == -(-n // 4) and samp[name][1] > 0, (name, n, samp[name])
