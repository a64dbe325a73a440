"""Pins the oracle to the reference itself (CPU, no GPU).

oracle/ref compiles the reference's own lib/asqtad_dslash_p.c,
lib/asqtad_invert_p.c, lib/invert_cg_p.c, lib/hisq_links_p.c,
lib/hisq_reunit*_p.c and lib/common_p.c, unmodified, against a
single-process CPU implementation of the QDP/QLA/QMP calls they make
(oracle/ref/qdp.h), into oracle/_ref/libqopref.so.  Two kinds of check:

  * against the committed fixture tests/golden/qopref_4x4x4x4.npz (the
    reference's outputs, written by tests/golden/make_qopref_golden.py):
    always run;
  * against the live library on more lattices and cases: run where
    oracle/_ref was built (the reference sources were present).

Bounds: link construction and Dslash agree to rounding (1e-13; HISQ links
to 1e-13 at the typical site and 1e-10 at the worst, the analytic U(3)
projection amplifying rounding where eigenvalues nearly coincide);
the FP64 solvers take the same iterations and restarts (the EVENODD
two-step solve within 2) and their solutions agree to 1e-9 relative;
the reference's single-precision build meets its 1e-10 target and agrees
with the FP64 oracle to 1e-4.
"""
import os

import numpy as np
import pytest

import oracle as O
import refqop as R
from helpers import rel_norm_err, half, eo_residual
from qopqdp_b200 import lattice as LT

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "qopref_4x4x4x4.npz")
live = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built (reference sources absent)")


def checksum(arrs):
    a = np.concatenate([np.asarray(x, dtype=np.float64).ravel() for x in arrs])
    w = np.cos(0.37 * np.arange(a.size))
    return np.array([float((a * a).sum()), float((a * w).sum())])


def close_ck(a, b, tol=1e-12):
    return np.all(np.abs(np.asarray(a) - np.asarray(b)) <= tol * (1 + np.abs(np.asarray(b))))


def maxdiff(a, b):
    return max(float(np.abs(np.asarray(x) - np.asarray(y)).max()) for x, y in zip(a, b))


# ---------------------------------------------------------------- fixture

@pytest.fixture(scope="module")
def gold():
    d = np.load(GOLD)
    L = tuple(int(x) for x in d["L"])
    U = LT.random_gauge(L, 0.3, 7)
    assert close_ck(checksum(U), d["gauge_ck"]), "gauge generator changed"
    G = O.Lattice(L).rephase_G(U, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
    src = LT.gaussian_vector(L, 41).reshape(-1, 6)
    assert close_ck(checksum([src]), d["src_ck"])
    return d, L, G, src


def test_golden_rephase_and_asqtad_links(gold):
    d, L, G, _ = gold
    assert close_ck(checksum(G), d["rephased_ck"])
    fat, lng = O.Lattice(L).make_imp_links(LT.ASQTAD_BENCH_COEFFS, G)
    assert close_ck(checksum(fat), d["asq_fat_ck"])
    assert close_ck(checksum(lng), d["asq_long_ck"])


def test_golden_asqtad_dslash_and_solves(gold):
    d, L, G, src = gold
    V = int(np.prod(L))
    fat, lng = O.Lattice(L).make_imp_links(LT.ASQTAD_BENCH_COEFFS, G)
    fo = O.Fla(O.Lattice(L), fat, lng)
    assert rel_norm_err(fo.dslash(0.1, src, 2, 2), d["asq_dslash_eoeo"]) < 1e-14
    assert rel_norm_err(fo.dslash(0.1, src, 0, 1), d["asq_dslash_e_o"]) < 1e-14
    ra = O.ResidArg(1e-20, 0, 0, 0, 0, 0)
    x, _ = fo.invert(0.1, src, O.InvertArg(1e9, 2000, 1000, 5, 0), ra)
    assert rel_norm_err(x[: V // 2], d["asq_invert_even"]) < 1e-9
    it, rs = d["asq_invert_even_iters"]
    assert abs(ra.final_iter - it) <= 2 and ra.final_restart == rs
    masses = [0.1, 0.2, 0.4]
    ras = [[O.ResidArg(1e-20, 0, 0, 0, 0, 0) for _ in masses]]
    xs, _ = fo.invert_multi([masses], [src], O.InvertArg(1e9, 2000, 1000, 5, 1), ras)
    for k in range(3):
        assert rel_norm_err(xs[0][k][V // 2:], d["asq_multi_odd"][k]) < 1e-9
        assert abs(ras[0][k].final_iter - d["asq_multi_odd_iters"][k]) <= 2


def test_golden_hisq_links_and_dslash(gold):
    d, L, G, src = gold
    hc = LT.hisq_coeff_vector(LT.hisq_bench_coeffs())
    fat, lng, W, _ = O.Lattice(L).hisq_links(hc, G, want_W=True)
    assert close_ck(checksum(fat), d["hisq_fat_ck"], 1e-11)
    assert close_ck(checksum(lng), d["hisq_long_ck"], 1e-11)
    assert close_ck(checksum(W), d["hisq_W_ck"], 1e-11)
    fo = O.Fla(O.Lattice(L), fat, lng)
    assert rel_norm_err(fo.dslash(0.05, src, 2, 2), d["hisq_dslash_eoeo"]) < 1e-13


def test_golden_forces(gold):
    """Fermion forces on a rough field with two filtered fat7 links: the
    oracle's asqtad force (ASVEC with one source, FNMAT with three) and its
    HISQ force (two Naik groups, the default force filter) equal the
    reference's outputs to rounding."""
    d, L, _, _ = gold
    V = int(np.prod(L))
    Ur = LT.random_gauge(L, 0.5, 2)
    assert close_ck(checksum(Ur), d["force_gauge_ck"])
    Gr = O.Lattice(L).rephase_G(Ur, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
    xs = [LT.gaussian_vector(L, 51 + i).reshape(V, 6) for i in range(3)]
    eps = [0.3, -0.2, 0.5]
    lat = O.Lattice(L)

    def agree(got, key, tol):
        ref = d[key]
        assert np.abs(np.stack(got) - ref).max() <= tol * np.abs(ref).max(), key

    agree(lat.asqtad_force(LT.ASQTAD_BENCH_COEFFS, Gr, eps[:1], xs[:1]), "force_asq_asvec", 1e-13)
    agree(lat.asqtad_force(LT.ASQTAD_BENCH_COEFFS, Gr, eps, xs), "force_asq_fnmat", 1e-13)
    hf = LT.hisq_coeff_vector(LT.hisq_bench_coeffs())
    hf[11], hf[12] = 0.3, -0.05
    agree(lat.hisq_force(hf, Gr, [0.0, 0.1], np.array(eps), xs, [2, 1]), "force_hisq", 1e-9)


# ---------------------------------------------------------------- live library

LIVE_L = [(4, 4, 4, 4), (4, 4, 4, 6), (8, 8, 8, 8), (6, 4, 4, 8)]


def _gauge(L, seed=5, eps=0.3):
    return LT.random_gauge(L, eps, seed)


@live
@pytest.mark.parametrize("L", LIVE_L)
@pytest.mark.parametrize("r0,bc", [((0, 0, 0, 0), (1, 1, 1, -1)), ((1, 0, 1, 1), (1, -1, 1j, -1)),
                                   ((0, 2, 0, 3), (1j, 1, -1, -1j))])
def test_live_rephase_bit_exact(L, r0, bc):
    U = _gauge(L)
    a = O.Lattice(L).rephase_G(U, r0, bc, (0, 1, 3, 7))
    b = R.rephase_G(L, U, r0, bc, (0, 1, 3, 7))
    assert maxdiff(a, b) == 0.0


@live
@pytest.mark.parametrize("L", LIVE_L[:2])
@pytest.mark.parametrize("coeffs", [LT.ASQTAD_BENCH_COEFFS, (0.625, -0.0625, 0.0104, -0.00130, -0.0625, -0.0417),
                                    (1.0, 0.0, 0.0, 0.0, 0.0, 0.0)])
@pytest.mark.parametrize("naik", [True, False])
def test_live_asqtad_links(L, coeffs, naik):
    G = O.Lattice(L).rephase_G(_gauge(L))
    fo, lo = O.Lattice(L).make_imp_links(coeffs, G, naik=naik)
    fr, lr = R.asqtad_links(L, coeffs, G, naik=naik)
    assert maxdiff(fo, fr) < 1e-13
    if naik:
        assert maxdiff(lo, lr) < 1e-13


@live
@pytest.mark.parametrize("L", LIVE_L[:2])
@pytest.mark.parametrize("eps", [(0.0,), (0.0, 0.1, -0.2)])
def test_live_hisq_links(L, eps):
    G = O.Lattice(L).rephase_G(_gauge(L, eps=0.5))
    hc = LT.hisq_coeff_vector(LT.hisq_bench_coeffs())
    hc[11], hc[12] = 0.3, -0.05
    so, dep_o = O.Lattice(L).hisq_links_naik(hc, G, eps)
    W_o = O.Lattice(L).hisq_links(hc, G, want_W=True)[2]
    sr, W_r, dep_r = R.hisq_links(L, hc, G, eps, want_deps=True)
    # the analytic U(3) projection (lib/hisq_reunit_utilities_p.c: the
    # eigenvalues of V^+V from a trigonometric cubic solution) amplifies
    # rounding at sites with nearly degenerate eigenvalues: a few sites reach
    # 1e-11 on O(1) links at eps 0.5; the typical site agrees to 1e-13
    def check(a, b):
        d = np.concatenate([np.abs(np.asarray(x) - np.asarray(y)).reshape(len(x), -1).max(axis=1)
                            for x, y in zip(a, b)])
        assert d.max() < 1e-10 and np.median(d) < 1e-13, (d.max(), np.median(d))
    for k in range(len(eps)):
        check(so[k][0], sr[k][0])
        check(so[k][1], sr[k][1])
    check(W_o, W_r)
    check(dep_o[0], dep_r[0])
    check(dep_o[1], dep_r[1])


def _ops(L, naik=True, seed=5):
    G = O.Lattice(L).rephase_G(_gauge(L, seed=seed))
    fat, lng = O.Lattice(L).make_imp_links(LT.ASQTAD_BENCH_COEFFS, G, naik=naik)
    return O.Fla(O.Lattice(L), fat, lng), fat, lng


@live
@pytest.mark.parametrize("L", LIVE_L)
@pytest.mark.parametrize("naik", [True, False])
def test_live_dslash_nine_cases(L, naik):
    fo, fat, lng = _ops(L, naik)
    fr = R.RefFla(L, fat, lng, R.D3)
    V = int(np.prod(L))
    x = np.random.default_rng(3).standard_normal((V, 6))
    prev = np.random.default_rng(4).standard_normal((V, 6))
    for eo_out in (0, 1, 2):
        for eo_in in (0, 1, 2):
            # out starts non-zero: sites outside eo_out keep their values
            a = fo.dslash(0.1, x, eo_out, eo_in, out=prev.copy())
            b = fr.dslash(0.1, x, eo_out, eo_in, out=prev.copy())
            assert rel_norm_err(a, b) < 1e-14, (eo_out, eo_in)


@live
@pytest.mark.parametrize("L", LIVE_L[:3])
@pytest.mark.parametrize("eo", [0, 1, 2])
def test_live_invert_fp64(L, eo):
    fo, fat, lng = _ops(L)
    fr = R.RefFla(L, fat, lng, R.D3)
    b = LT.gaussian_vector(L, 40 + eo).reshape(-1, 6)
    ia = O.InvertArg(1e9, 800, 300, 5, eo)
    ra_o, ra_r = O.ResidArg(1e-20, 0, 0, 0, 0, 0), O.ResidArg(1e-20, 0, 0, 0, 0, 0)
    xo, _ = fo.invert(0.1, b, ia, ra_o)
    xr, _ = fr.invert(0.1, b, ia, ra_r)
    assert rel_norm_err(half(xo, L, eo), half(xr, L, eo)) < 1e-9
    # the oracle's OpenMP reductions round differently from the serial shim
    assert abs(ra_o.final_iter - ra_r.final_iter) <= (3 if eo == 2 else 2)
    assert ra_o.final_restart == ra_r.final_restart
    assert ra_r.final_rsq <= 1e-20 and ra_o.final_rsq <= 1e-20


@live
@pytest.mark.parametrize("eo", [0, 1])
def test_live_invert_single_precision_build(eo):
    L = (4, 4, 4, 6)
    fo, fat, lng = _ops(L)
    fr = R.RefFla(L, fat, lng, R.F3)
    b = LT.gaussian_vector(L, 50 + eo).reshape(-1, 6)
    ra = O.ResidArg(1e-10, 0, 0, 0, 0, 0)
    xr, _ = fr.invert(0.1, b, O.InvertArg(1e9, 800, 300, 5, eo), ra)
    assert eo_residual(fo, 0.1, xr, b, L, eo) <= 1e-10 * 50
    xo, _ = fo.invert(0.1, b, O.InvertArg(1e9, 800, 300, 5, eo), O.ResidArg(1e-20, 0, 0, 0, 0, 0))
    assert rel_norm_err(half(xr, L, eo), half(xo, L, eo)) < 1e-4


@live
@pytest.mark.parametrize("eo", [0, 1, 2])
@pytest.mark.parametrize("restart", [200, 500])
def test_live_invert_multi_one_source(eo, restart):
    """One source, three masses.  EVEN / ODD: every mass converges; the
    iteration counts agree to a few percent (whether the true residual at a
    CG stop lies just above or below rsqmin, and so whether one more restart
    runs, depends on rounding).  EVENODD, which the reference warns it does
    not support: its solve stops when the heaviest mass converges, leaving
    the lighter ones short of rsqmin; the oracle stops at the same iteration
    with the same residuals."""
    L = (4, 4, 4, 6)
    fo, fat, lng = _ops(L)
    fr = R.RefFla(L, fat, lng, R.D3)
    masses = [[0.1, 0.2, 0.4]]
    ins = [LT.gaussian_vector(L, 60).reshape(-1, 6)]
    ra_o = [[O.ResidArg(1e-20, 0, 0, 0, 0, 0) for _ in masses[0]]]
    ra_r = [[O.ResidArg(1e-20, 0, 0, 0, 0, 0) for _ in masses[0]]]
    ia = O.InvertArg(1e9, 1500, restart, 5, eo)
    xo, _ = fo.invert_multi(masses, ins, ia, ra_o)
    xr, _ = fr.invert_multi(masses, ins, ia, ra_r)
    for k in range(3):
        a, b = ra_o[0][k], ra_r[0][k]
        if eo == 2:
            assert abs(a.final_iter - b.final_iter) <= 2
            assert abs(a.final_rsq - b.final_rsq) <= 0.01 * b.final_rsq + 1e-22, (k, a.final_rsq, b.final_rsq)
            assert rel_norm_err(half(xo[0][k], L, eo), half(xr[0][k], L, eo)) < 1e-5, k
        else:
            assert abs(a.final_iter - b.final_iter) <= 0.05 * b.final_iter + 2, (k, a.final_iter, b.final_iter)
            assert a.final_rsq <= 1e-20 and b.final_rsq <= 1e-20
            assert rel_norm_err(half(xo[0][k], L, eo), half(xr[0][k], L, eo)) < 1e-9, k


@live
@pytest.mark.parametrize("eo", [0, 1, 2])
def test_live_invert_multi_two_sources(eo):
    """Two sources with different mass lists: the reference flattens them
    into one solve_multi (EVEN / ODD), whose shifted CG runs on the least
    converged system's residual and reaches the others through restarts,
    or (EVENODD, which it warns is unsupported) solves each source's masses
    in turn.  With max_restarts = 5 the flattened solve stops before
    converging; the oracle must stop at the same iteration and restart with
    the same residuals."""
    L = (4, 4, 4, 6)
    fo, fat, lng = _ops(L)
    fr = R.RefFla(L, fat, lng, R.D3)
    masses = [[0.1, 0.2, 0.4], [0.05, 0.3]]
    ins = [LT.gaussian_vector(L, 60 + s).reshape(-1, 6) for s in range(2)]
    ra_o = [[O.ResidArg(1e-20, 0, 0, 0, 0, 0) for _ in m] for m in masses]
    ra_r = [[O.ResidArg(1e-20, 0, 0, 0, 0, 0) for _ in m] for m in masses]
    ia = O.InvertArg(1e9, 1500, 500, 5, eo)
    xo, _ = fo.invert_multi(masses, ins, ia, ra_o)
    xr, _ = fr.invert_multi(masses, ins, ia, ra_r)
    for s in range(2):
        for k in range(len(masses[s])):
            a, b = ra_o[s][k], ra_r[s][k]
            assert abs(a.final_iter - b.final_iter) <= 2 and a.final_restart == b.final_restart, (s, k)
            # unconverged residuals after hundreds of iterations: rounding
            # (the oracle's reduction order follows its thread count) moves
            # them by up to tens of percent, not by orders of magnitude
            assert abs(a.final_rsq - b.final_rsq) <= 0.25 * b.final_rsq + 1e-22, (s, k, a.final_rsq, b.final_rsq)
            assert rel_norm_err(half(xo[s][k], L, eo), half(xr[s][k], L, eo)) < 1e-3, (s, k)


# ---------------------------------------------------------------- forces

@live
@pytest.mark.parametrize("coeffs", [LT.ASQTAD_BENCH_COEFFS, (0.625, -0.0625, 0.0104, -0.00130, -0.0625, -0.0417)])
@pytest.mark.parametrize("nsrc,fsm", [(1, 2), (1, 0), (3, 2), (3, 4)])
def test_live_asqtad_force(coeffs, nsrc, fsm):
    """QOP_D3_asqtad_force_multi_qdp with the reference's algorithm choice
    (ASVEC for nsrc < fnmat_src_min, FNMAT otherwise), accumulated into a
    force field that is not anti-Hermitian: the oracle agrees to rounding in
    all four cases (ASVEC stores TA(force + C), its contribution half of
    FNMAT's)."""
    L = (4, 4, 4, 6)
    V = int(np.prod(L))
    G = O.Lattice(L).rephase_G(_gauge(L))
    rng = np.random.default_rng(9)
    xs = [rng.standard_normal((V, 6)) for _ in range(nsrc)]
    eps = [0.3, -0.2, 0.5][:nsrc]
    f0 = [rng.standard_normal((V, 3, 3, 2)) * 0.1 for _ in range(4)]
    fo = O.Lattice(L).asqtad_force(coeffs, G, eps, xs, force=f0, fnmat_src_min=fsm)
    fr = R.asqtad_force(L, coeffs, G, eps, xs, force=f0, fnmat_src_min=fsm)
    scale = max(float(np.abs(a).max()) for a in fo)
    assert maxdiff(fo, fr) < 1e-13 * scale


@live
@pytest.mark.parametrize("coeffs", [LT.ASQTAD_BENCH_COEFFS, (0.625, -0.0625, 0.0104, -0.00130, -0.0625, -0.0417)])
def test_live_asqtad_deriv(coeffs):
    """The derivative field itself (QOP_D3_asqtad_deriv): the oracle's
    reverse sweep plus the reference's Lepage term (lepage_rep) equals the
    reference's field to rounding; the general-complex derivative (pinned by
    finite differences in test_oracle.py) differs from it by U H with H
    Hermitian, which the force projection TA(U D^+) removes."""
    L = (4, 4, 4, 6)
    V = int(np.prod(L))
    G = O.Lattice(L).rephase_G(_gauge(L, eps=0.5))
    rng = np.random.default_rng(2)
    mF = [rng.standard_normal((V, 3, 3, 2)) for _ in range(4)]
    mN = [rng.standard_normal((V, 3, 3, 2)) for _ in range(4)]
    cz = lambda a: a[..., 0] + 1j * a[..., 1]
    dr = R.asqtad_deriv(L, coeffs, G, mF, mN)
    do = O.Lattice(L).asqtad_deriv(coeffs, G, mF, mN, lepage_rep=True)
    scale = max(float(np.abs(a).max()) for a in dr)
    assert maxdiff(do, dr) < 1e-13 * scale
    dg = O.Lattice(L).asqtad_deriv(coeffs, G, mF, mN)
    assert maxdiff(dg, dr) > 1e-3 * scale               # the Lepage term is there
    for mu in range(4):
        x = np.einsum("sij,skj->sik", cz(G[mu]), np.conj(cz(dr[mu]) - cz(dg[mu])))   # U (D_ref - D_general)^+
        assert np.abs(x - np.conj(np.swapaxes(x, 1, 2))).max() < 1e-12 * scale


@live
@pytest.mark.parametrize("eps_g,ff", [(0.2, 5e-5), (0.5, 0.0)])
@pytest.mark.parametrize("eps_naik", [(0.0,), (0.0, 0.1)])
def test_live_hisq_force(eps_g, ff, eps_naik):
    """QOP_D3_hisq_force_multi_qdp (U(3) projection, the RATIONAL force
    branch): the oracle agrees to rounding on a smooth gauge field (every
    fat7 link's V^+V eigenvalues above the 5e-5 default filter) and on a
    rough one with the filter off (force_filter 0)."""
    L = (4, 4, 4, 6)
    V = int(np.prod(L))
    G = O.Lattice(L).rephase_G(_gauge(L, eps=eps_g))
    rng = np.random.default_rng(9)
    xs = [rng.standard_normal((V, 6)) for _ in range(3)]
    res = [0.3, -0.2, 0.5]
    n_orders = [3] if len(eps_naik) == 1 else [2, 1]
    hc = LT.hisq_coeff_vector(LT.hisq_bench_coeffs(), force_filter=ff)
    hc[11], hc[12] = 0.3, -0.05
    fo = O.Lattice(L).hisq_force(hc, G, list(eps_naik), np.array(res), xs, n_orders)
    fr = R.hisq_force(L, hc, G, list(eps_naik), res, xs, n_orders)
    scale = max(float(np.abs(a).max()) for a in fo)
    assert maxdiff(fo, fr) < 1e-9 * scale, (maxdiff(fo, fr), scale)


@live
def test_live_force_filter_per_link():
    """At a filtered link (V^+V eigenvalue below force_filter) the
    reference's derivative tensors are those of V (V^+V + ff)^-1/2, and its
    chain rule equals the oracle's adjoint with the filter; elsewhere the
    filter does nothing."""
    L = (4, 4, 4, 6)
    G = O.Lattice(L).rephase_G(_gauge(L, eps=0.5))
    hc = LT.hisq_coeff_vector(LT.hisq_bench_coeffs())
    Vl, _ = O.Lattice(L).make_imp_links([hc[0], hc[1], hc[2], hc[3], 0.0, 0.0], G, naik=False)
    cz = lambda a: a[..., 0] + 1j * a[..., 1]
    Vs = np.concatenate([cz(v) for v in Vl])
    wmin = np.linalg.eigvalsh(np.einsum("sji,sjk->sik", Vs.conj(), Vs)).min(axis=1)
    bad = int(np.argmin(wmin))
    assert wmin[bad] < 5e-5 <= np.sort(wmin)[1]     # one filtered link on this field

    def W(X, e):
        w, Z = np.linalg.eigh(X.conj().T @ X + e * np.eye(3))
        return X @ (Z @ np.diag(w ** -0.5) @ Z.conj().T)

    def adj(X, GW, e):
        w, Z = np.linalg.eigh(X.conj().T @ X)
        if e > 0 and w.min() < e:
            w = w + e
        s = np.sqrt(w)
        At = (Z.conj().T @ (X.conj().T @ GW) @ Z) * (-1.0 / (s[:, None] * s[None, :] * (s[:, None] + s[None, :])))
        B = Z @ At @ Z.conj().T
        return GW @ (Z @ np.diag(1 / s) @ Z.conj().T) + X @ (B + B.conj().T)

    rng = np.random.default_rng(4)
    for k in (bad, 10):
        X = Vs[k]
        dw, dwd, ff = R.u3_der(L, X)
        assert ff == (k == bad)
        h = 1e-7
        for m in range(3):
            for n in range(3):
                E = np.zeros((3, 3), complex)
                E[m, n] = 1
                fd = 0.5 * ((W(X + h * E, 5e-5 if ff else 0) - W(X - h * E, 5e-5 if ff else 0))
                            - 1j * (W(X + 1j * h * E, 5e-5 if ff else 0) - W(X - 1j * h * E, 5e-5 if ff else 0))) / (2 * h)
                assert np.abs(dw[:, :, m, n] - fd).max() < 1e-5 * max(1.0, np.abs(fd).max())
        F = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
        new = np.einsum("ijmn,ji->nm", dw, F) + np.einsum("ijmn,ji->nm", dwd, F.conj().T)
        mine = adj(X, F.conj().T, 5e-5).conj().T
        assert np.abs(new - mine).max() < 1e-8 * np.abs(new).max()


@live
@pytest.mark.parametrize("eps_naik", [(0.0,), (0.0, 0.1)])
def test_live_hisq_force_filtered(eps_naik):
    """The whole HISQ force on a rough field with one filtered link and the
    default filter: the W-level derivative that the filtered U(3) adjoint
    receives carries the reference's Lepage term (test_live_asqtad_deriv),
    which that adjoint does not remove, so the oracle matches the reference
    on every link, the ~140 around the filtered one included."""
    L = (4, 4, 4, 6)
    V = int(np.prod(L))
    G = O.Lattice(L).rephase_G(_gauge(L, eps=0.5))
    hc = LT.hisq_coeff_vector(LT.hisq_bench_coeffs())
    Vl, _ = O.Lattice(L).make_imp_links([hc[0], hc[1], hc[2], hc[3], 0.0, 0.0], G, naik=False)
    cz = lambda a: a[..., 0] + 1j * a[..., 1]
    Vs = np.concatenate([cz(v) for v in Vl])
    wmin = np.linalg.eigvalsh(np.einsum("sji,sjk->sik", Vs.conj(), Vs)).min(axis=1)
    assert (wmin < 5e-5).sum() == 1                 # one filtered link on this field
    rng = np.random.default_rng(9)
    xs = [rng.standard_normal((V, 6)) for _ in range(3)]
    res = [0.3, -0.2, 0.5]
    n_orders = [3] if len(eps_naik) == 1 else [2, 1]
    hc[11], hc[12] = 0.3, -0.05
    fo = O.Lattice(L).hisq_force(hc, G, list(eps_naik), np.array(res), xs, n_orders)
    fr = R.hisq_force(L, hc, G, list(eps_naik), res, xs, n_orders)
    scale = max(float(np.abs(a).max()) for a in fo)
    assert maxdiff(fo, fr) < 1e-9 * scale, (maxdiff(fo, fr), scale)
