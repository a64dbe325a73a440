"""Link construction and handle round trips on the device vs the oracle:
rephase_G (lib/common_p.c:455-526), asqtad_create_L_from_G (make_imp_links,
lib/asqtad_dslash_p.c:458-633), hisq_create_L_from_G (fat7 -> U(3) ->
asqtad, lib/hisq_links_p.c:62-256), extract/load L (x2 / x1/2 convention,
:915-938) and rephase_L (:1447-1482)."""
import numpy as np
import pytest

import oracle as O
from conftest import gpu_lattice
from helpers import gauge, asqtad_links, hisq_links, site_rel_err, rel_norm_err
from qopqdp_b200 import lattice as LT
from qopqdp_b200.qop import QOP_info_t

pytestmark = pytest.mark.gpu

L = (4, 4, 4, 8)
V = int(np.prod(L))


def test_rephase_G_matches_oracle():
    q = gpu_lattice(L, "D")
    U = LT.random_gauge(L, 0.3, 7)
    g = q.create_G(U)
    q.rephase_G(g, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
    got = q.extract_G(g, V)
    ref = O.Lattice(L).rephase_G(U)
    for mu in range(4):
        assert np.array_equal(got[mu], ref[mu])
    q.destroy_G(g)


@pytest.mark.parametrize("prec", ["D", "F"])
def test_create_L_from_G_matches_make_imp_links(prec):
    q = gpu_lattice(L, prec)
    U = [np.asarray(u, dtype=q.dtype) for u in gauge(L, 0.3, 7)]
    g = q.create_G(U)
    info = QOP_info_t()
    fla = q.create_L_from_G(LT.ASQTAD_BENCH_COEFFS, g, info)
    assert info.status == 0 and info.final_flop == 61632.0 * V
    fat, lng = q.extract_L(fla, V)
    rfat, rlng = O.Lattice(L).make_imp_links(LT.ASQTAD_BENCH_COEFFS, [u.astype(np.float64) for u in U])
    tol = 1e-13 if prec == "D" else 2e-6
    for mu in range(4):
        assert site_rel_err(fat[mu], rfat[mu]) <= tol
        assert site_rel_err(lng[mu], rlng[mu]) <= tol
    q.destroy_L(fla)
    q.destroy_G(g)


@pytest.mark.parametrize("prec", ["D", "F"])
def test_hisq_links_match_oracle(prec):
    q = gpu_lattice(L, prec)
    U = [np.asarray(u, dtype=q.dtype) for u in gauge(L, 0.5, 9)]
    g = q.create_G(U)
    info = QOP_info_t()
    h = q.hisq_create_L_from_G(LT.hisq_bench_coeffs(), g, info)
    assert info.status == 0
    fla = q.hisq_asqtad_links(h, 0)
    fat, lng = q.extract_L(fla, V)
    rfat, rlng, _, nsvd = O.Lattice(L).hisq_links(LT.hisq_coeff_vector(LT.hisq_bench_coeffs()),
                                                  [u.astype(np.float64) for u in U])
    tol = 1e-10 if prec == "D" else 2e-6   # analytic U(3) step is ill-conditioned at some sites
    for mu in range(4):
        assert site_rel_err(fat[mu], rfat[mu]) <= tol
        assert site_rel_err(lng[mu], rlng[mu]) <= tol
    q.hisq_destroy_L(h)
    q.destroy_G(g)


@pytest.mark.parametrize("prec", ["D", "F"])
def test_hisq_eps_naik_link_sets_match_oracle(prec):
    """n_naiks = 3 (lib/hisq_links_p.c:182-243): fn[0] = asqtad(W), fn[k] =
    eps_k x difference links + fn[0], and the difference links themselves
    (want_deps), each compared link by link with the oracle."""
    q = gpu_lattice(L, prec)
    U = [np.asarray(u, dtype=q.dtype) for u in gauge(L, 0.5, 9)]
    g = q.create_G(U)
    hc = LT.hisq_bench_coeffs()
    hc.n_naiks = 3
    eps = [0.0, -0.0632, 0.041]
    for k, e in enumerate(eps):
        hc.eps_naik[k] = e
    hc.difference_one_link, hc.difference_naik = 0.0375, -0.0413
    assert q.set_hisq_opts(want_deps=1) == 0
    info = QOP_info_t()
    h = q.hisq_create_L_from_G(hc, g, info)
    assert info.status == 0
    sets, (dfat, dlng) = O.Lattice(L).hisq_links_naik(LT.hisq_coeff_vector(hc), [u.astype(np.float64) for u in U],
                                                      eps)
    tol = 1e-10 if prec == "D" else 2e-6
    for k in range(3):
        fat, lng = q.extract_L(q.hisq_asqtad_links(h, k), V)
        for mu in range(4):
            assert site_rel_err(fat[mu], sets[k][0][mu]) <= tol, (k, mu)
            assert site_rel_err(lng[mu], sets[k][1][mu]) <= tol, (k, mu)
    deps = q.f("get_asqtad_deps_links_from_hisq")(h)
    assert deps
    fat, lng = q.extract_L(deps, V)
    for mu in range(4):
        assert site_rel_err(fat[mu], dfat[mu]) <= tol and site_rel_err(lng[mu], dlng[mu]) <= tol
    assert q.set_hisq_opts(want_deps=0) == 0
    q.hisq_destroy_L(h)
    q.destroy_G(g)


@pytest.mark.parametrize("prec", ["D", "F"])
def test_extract_load_roundtrip_and_scaling(prec):
    q = gpu_lattice(L, prec)
    fat, lng = asqtad_links(L, 0.3, 7)
    fat = [np.asarray(a, dtype=q.dtype) for a in fat]
    lng = [np.asarray(a, dtype=q.dtype) for a in lng]
    fla = q.create_L_from_raw(fat, lng)
    ef, el = q.extract_L(fla, V)
    for mu in range(4):      # x1/2 on load, x2 on extract: exact in binary
        assert np.array_equal(ef[mu], fat[mu]) and np.array_equal(el[mu], lng[mu])
    # load_L_from_raw on the odd half keeps the even half
    fat2 = [(2 * a).astype(q.dtype) for a in fat]
    q.load_L_from_raw(fla, fat2, lng, 1)
    ef, _ = q.extract_L(fla, V)
    for mu in range(4):
        assert np.array_equal(ef[mu][: V // 2], fat[mu][: V // 2])
        assert np.array_equal(ef[mu][V // 2:], fat2[mu][V // 2:])
    q.destroy_L(fla)


def test_rephase_L_matches_oracle_semantics():
    """rephase_L on links equals rephasing the raw links the reference way."""
    q = gpu_lattice(L, "D")
    fat, lng = asqtad_links(L, 0.3, 7)
    fla = q.create_L_from_raw(fat, lng)
    r0 = (1, 0, 2, 3)
    q.rephase_L(fla, r0, (1, 1, 1, -1), (0, 1, 3, 7))
    ef, el = q.extract_L(fla, V)
    xs = LT.raw_coords(L)
    for mu in range(4):
        n = L[3]
        rs = (xs[:, 3] + n - r0[3]) % n
        sgn = np.zeros(V, dtype=np.int64)
        for j in range(4):
            if (LT.BENCH_SIGNMASK[mu] >> j) & 1:
                sgn += (xs[:, j] + L[j] - r0[j]) % L[j]
        s = np.where(sgn & 1, -1.0, 1.0)
        ff = np.where(rs == n - 1, -1.0, 1.0) if mu == 3 else 1.0
        fl = np.where(rs >= n - 3, -1.0, 1.0) if mu == 3 else 1.0
        np.testing.assert_array_equal(ef[mu], fat[mu] * (s * ff)[:, None, None, None])
        np.testing.assert_array_equal(el[mu], lng[mu] * (s * fl)[:, None, None, None])
    # the double-stored backward links follow: dslash equals the oracle's
    fo = O.Fla(O.Lattice(L), ef, el)
    src = LT.gaussian_vector(L, 4)
    hi, ho = q.create_V(src), q.create_V(np.zeros_like(src))
    q.dslash(fla, 0.1, ho, hi, 2, 2)
    assert site_rel_err(q.extract_V(ho, V), fo.dslash(0.1, src, 2, 2)) <= 1e-13
    q.destroy_V(hi)
    q.destroy_V(ho)
    q.destroy_L(fla)


def test_fd_link_copy():
    q = gpu_lattice(L, "D")
    fat, lng = asqtad_links(L, 0.3, 7)
    fla = q.create_L_from_raw(fat, lng)
    f32 = q.lib.QOP_FD3_asqtad_create_L_from_L(fla)
    assert f32
    from qopqdp_b200.qop import Qop
    qf = Qop("F")
    ef, el = qf.extract_L(f32, V)
    for mu in range(4):
        assert rel_norm_err(ef[mu], fat[mu]) < 1e-7
    qf.destroy_L(f32)
    q.destroy_L(fla)
