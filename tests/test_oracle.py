"""CPU tests of the oracle (no GPU).

The reference ships no golden vectors and cannot be built here (it needs the
external QDP/C, QLA and QMP libraries), so the oracle is pinned to the
reference's own tests and to the identities the algorithm guarantees:
  * examples/asqtad_test.c:37-81 check_op: Dslash rebuilt from the unscaled
    links with plain shifts agrees to <= 1e-10 (squared, relative);
  * examples/asqtad_test.c:84-130 check_resids: the eo solve's true residual
    |in - (1/m)(m^2 - D D) out|^2/|in|^2 meets rsqmin;
  * layout (lib/layout_user.c:237-258), rephase (lib/common_p.c:455-526),
    U(3) projection (W^+W = 1), gauge covariance, anti-hermiticity of the hop.
"""
import numpy as np
import pytest

import oracle as O
from helpers import gauge, asqtad_links, hisq_links, eo_residual, full_residual, half
from qopqdp_b200 import lattice as LT

LATTICES = [(4, 4, 4, 4), (4, 4, 4, 8), (6, 4, 4, 4)]


@pytest.mark.parametrize("L", LATTICES)
def test_raw_index_matches_layout_formula(L):
    lat = O.Lattice(L)
    xs = LT.raw_coords(L)
    V = int(np.prod(L))
    assert sorted(LT.raw_index(L, xs)) == list(range(V))
    import ctypes as C
    for idx in (0, 1, V // 2 - 1, V // 2, V - 1):
        x = (C.c_int * 4)(*[int(v) for v in xs[idx]])
        assert O.lib().or_raw_index(lat.h, x) == idx
    # even sites first
    assert (xs[: V // 2].sum(axis=1) % 2 == 0).all() and (xs[V // 2:].sum(axis=1) % 2 == 1).all()


@pytest.mark.parametrize("L", LATTICES)
@pytest.mark.parametrize("naik", [True, False])
def test_check_op_identity(L, naik):
    fat, lng = asqtad_links(L, 0.3, 7, naik)
    fo = O.Fla(O.Lattice(L), fat, lng)
    src = LT.gaussian_vector(L, 1)
    for m in (0.1, 0.0):
        d2 = fo.check_op(m, src)
        assert d2 <= 1e-28, d2          # the reference test demands <= 1e-10


def test_check_op_hisq():
    L = (4, 4, 4, 8)
    fat, lng, W, _ = hisq_links(L, 0.5, 9)
    fo = O.Fla(O.Lattice(L), fat, lng)
    assert fo.check_op(0.05, LT.gaussian_vector(L, 2)) <= 1e-28
    # the analytic projection (hisq_reunit_utilities_p.c:99-297) loses a few
    # digits where fat7 links have nearly degenerate V^+V eigenvalues
    for mu in range(4):
        w = LT.to_complex(W[mu])
        assert np.abs(np.einsum("vij,vkj->vik", w, w.conj()) - np.eye(3)).max() < 1e-9


def test_u3_projection_fixes_unitary_and_polar_factor():
    rng = np.random.default_rng(0)
    import ctypes as C
    for _ in range(20):
        a = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
        Vr = LT.from_complex(a).ravel()
        Wr = np.zeros(18)
        O.lib().or_u3_un_analytic(O._p(Vr), O._p(Wr), 1, 1e-8, 1e-8)
        W = LT.to_complex(Wr.reshape(3, 3, 2))
        u, s, vh = np.linalg.svd(a)
        assert np.abs(W - u @ vh).max() < 1e-10        # polar factor V (V^+V)^-1/2
        Wr2 = np.zeros(18)
        O.lib().or_u3_un_analytic(O._p(LT.from_complex(W).ravel()), O._p(Wr2), 1, 1e-8, 1e-8)
        assert np.abs(LT.to_complex(Wr2.reshape(3, 3, 2)) - W).max() < 1e-12
    # near-singular input takes the eigen-decomposition fallback
    a = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
    a[2] = a[0] * (1 + 1e-9)
    Wr = np.zeros(18)
    assert O.lib().or_u3_un_analytic(O._p(LT.from_complex(a).ravel()), O._p(Wr), 1, 1e-8, 1e-8) == 1


def test_rephase_G_signs_and_boundary():
    L = (4, 4, 4, 8)
    U = LT.random_gauge(L, 0.3, 3)
    R = O.Lattice(L).rephase_G(U, (0, 0, 0, 0), (1, 1, 1, -1), (0, 1, 3, 7))
    xs = LT.raw_coords(L)
    for mu, mask in enumerate((0, 1, 3, 7)):
        s = np.zeros(len(xs), dtype=np.int64)
        for j in range(4):
            if (mask >> j) & 1:
                s += xs[:, j]
        f = np.where(s % 2 == 1, -1.0, 1.0)
        if mu == 3:
            f = f * np.where(xs[:, 3] == L[3] - 1, -1.0, 1.0)
        np.testing.assert_array_equal(R[mu], U[mu] * f[:, None, None, None])


def test_hop_is_antihermitian_and_gauge_covariant():
    L = (4, 4, 4, 4)
    fat, lng = asqtad_links(L, 0.3, 7)
    fo = O.Fla(O.Lattice(L), fat, lng)
    x = LT.to_complex(LT.gaussian_vector(L, 5))
    y = LT.to_complex(LT.gaussian_vector(L, 6))
    Dy = LT.to_complex(fo.dslash(0.0, LT.from_complex(y), 2, 2))
    Dx = LT.to_complex(fo.dslash(0.0, LT.from_complex(x), 2, 2))
    lhs = np.vdot(x, Dy)
    rhs = -np.vdot(Dx, y)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    # gauge covariance: U -> g(x) U g(x+mu)^+ on the base links, psi -> g psi
    Ug = [LT.to_complex(u) for u in gauge(L, 0.3, 7)]
    gx = LT.to_complex(LT.random_gauge(L, 1.0, 99)[0])
    xs = LT.raw_coords(L)
    Ut = []
    for mu in range(4):
        y_ = xs.copy()
        y_[:, mu] = (y_[:, mu] + 1) % L[mu]
        nb = LT.raw_index(L, y_)
        Ut.append(LT.from_complex(np.einsum("vij,vjk,vlk->vil", gx, Ug[mu], gx[nb].conj())))
    lat = O.Lattice(L)
    f2, l2 = lat.make_imp_links(LT.ASQTAD_BENCH_COEFFS, Ut)
    fo2 = O.Fla(lat, f2, l2)
    psi = LT.to_complex(LT.gaussian_vector(L, 8))
    a = LT.to_complex(fo2.dslash(0.1, LT.from_complex(np.einsum("vij,vj->vi", gx, psi)), 2, 2))
    b = np.einsum("vij,vj->vi", gx, LT.to_complex(fo.dslash(0.1, LT.from_complex(psi), 2, 2)))
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


@pytest.mark.parametrize("eo", [0, 1])
def test_check_resids_eo_solve(eo):
    L = (4, 4, 4, 8)
    fat, lng = asqtad_links(L, 0.3, 7)
    fo = O.Fla(O.Lattice(L), fat, lng)
    src = LT.gaussian_vector(L, 20)
    ia, ra = O.InvertArg(1e9, 2000, 1000, 5, eo), O.ResidArg(1e-20, 0, 0, 0, 0, 0)
    out, flop = fo.invert(0.1, src, ia, ra)
    true = eo_residual(fo, 0.1, out, src, L, eo)
    assert true <= 1e-20 * 1.01 and abs(true - ra.final_rsq) <= 1e-3 * true
    assert not half(out, L, 1 - eo).any()
    # restarting from the solution needs (almost) no iterations
    ra2 = O.ResidArg(1e-20, 0, 0, 0, 0, 0)
    fo.invert(0.1, src, O.InvertArg(1e9, 2000, 1000, 5, eo), ra2, out=out)
    assert ra2.final_iter <= 2
    assert flop == 0.5 * (60 + 2 * 8 * 9 * 16) * ra.final_iter * int(np.prod(L))


def test_evenodd_solve_and_multimass():
    L = (4, 4, 4, 8)
    fat, lng, _, _ = hisq_links(L, 0.5, 9)
    fo = O.Fla(O.Lattice(L), fat, lng)
    src = LT.gaussian_vector(L, 21)
    ra = O.ResidArg(1e-18, 0, 0, 0, 0, 0)
    out, _ = fo.invert(0.05, src, O.InvertArg(1e9, 2000, 1000, 5, 2), ra)
    assert full_residual(fo, 0.05, out, src) <= 1e-18 * 1.01
    ms = [0.02, 0.05, 0.2]
    ras = [[O.ResidArg(1e-18, 0, 0, 0, 0, 0) for _ in ms]]
    outs, _ = fo.invert_multi([ms], [src], O.InvertArg(1e9, 8000, 1000, 20, 0), ras)
    for j, m in enumerate(ms):
        assert eo_residual(fo, m, outs[0][j], src, L, 0) <= 1e-18 * 1.05


# ---------------------------------------------------------------- fermion force
def _shift(L, mu, d):
    X = LT.raw_coords(L)
    Y = X.copy()
    Y[:, mu] = (Y[:, mu] + d) % L[mu]
    return LT.raw_index(L, Y)


def _cgauss(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _E(lat, coef, U, midF, midN):
    fat, lng = lat.make_imp_links(coef, U, naik=True)
    e = 0.0
    for mu in range(4):
        e += np.sum(np.conj(LT.to_complex(midF[mu])) * LT.to_complex(fat[mu])).real
        e += np.sum(np.conj(LT.to_complex(midN[mu])) * LT.to_complex(lng[mu])).real
    return e


@pytest.mark.parametrize("coef", [(1.0, 0.1, 0.1, 0.1, 0.1, 0.1), (0.7, -0.23, 0.31, -0.17, 0.29, -0.13)])
def test_asqtad_deriv_is_the_derivative_of_the_smeared_links(coef):
    """deriv = dE/dU for E = Re sum tr[midF^+ fat + midN^+ long], fat/long from
    make_imp_links (one-link, 3-, 5-, 7-staple, Lepage and Naik terms):
    central finite differences along random directions agree to 1e-7."""
    L = (4, 4, 4, 6)
    V = int(np.prod(L))
    lat = O.Lattice(L)
    rng = np.random.default_rng(3)
    U = [np.asarray(u) for u in gauge(L, 0.3, 5)]
    midF = [LT.from_complex(_cgauss(rng, (V, 3, 3))) for _ in range(4)]
    midN = [LT.from_complex(_cgauss(rng, (V, 3, 3))) for _ in range(4)]
    der = lat.asqtad_deriv(coef, U, midF, midN)
    for trial in range(2):
        dU = [_cgauss(rng, (V, 3, 3)) for _ in range(4)]
        h = 1e-5
        Up = [LT.from_complex(LT.to_complex(U[m]) + h * dU[m]) for m in range(4)]
        Um = [LT.from_complex(LT.to_complex(U[m]) - h * dU[m]) for m in range(4)]
        fd = (_E(lat, coef, Up, midF, midN) - _E(lat, coef, Um, midF, midN)) / (2 * h)
        an = sum(np.sum(np.conj(LT.to_complex(der[m])) * dU[m]).real for m in range(4))
        assert abs(fd - an) <= 1e-7 * abs(an), (fd, an)


def test_asqtad_force_outer_products_and_projection():
    """force_mu = -2 TA(U_mu deriv_mu^+) with deriv from the outer products
    midF_mu(x) = -s(x) sum_i eps_i x_i(x) x_i(x+mu)^+ (x+3mu for Naik),
    s = -1 on odd sites (lib/asqtad_force_fnmat_p.c:4-43, :491-546); the result
    is traceless anti-Hermitian and accumulates into the force field."""
    L = (4, 4, 4, 6)
    V = int(np.prod(L))
    lat = O.Lattice(L)
    coef = (1.0, 0.1, 0.1, 0.1, 0.1, 0.1)
    U = [np.asarray(u) for u in gauge(L, 0.3, 5)]
    xs = [LT.gaussian_vector(L, 70 + i) for i in range(2)]
    eps = [0.7, -0.4]
    f0 = [LT.from_complex(_cgauss(np.random.default_rng(1), (V, 3, 3))) for _ in range(4)]
    F = lat.asqtad_force(coef, U, eps, xs, force=f0)
    sgn = np.where(LT.parity_mask(L), -1.0, 1.0)
    midF, midN = [], []
    for mu in range(4):
        mf = np.zeros((V, 3, 3), complex)
        mn = np.zeros((V, 3, 3), complex)
        for e, x in zip(eps, xs):
            xc = LT.to_complex(x)
            mf += e * np.einsum("va,vb->vab", xc, np.conj(xc[_shift(L, mu, 1)]))
            mn += e * np.einsum("va,vb->vab", xc, np.conj(xc[_shift(L, mu, 3)]))
        midF.append(LT.from_complex(sgn[:, None, None] * mf))
        midN.append(LT.from_complex(sgn[:, None, None] * mn))
    der = lat.asqtad_deriv(coef, U, midF, midN)
    for mu in range(4):
        A = LT.to_complex(U[mu]) @ np.conj(np.transpose(LT.to_complex(der[mu]), (0, 2, 1)))
        T = 0.5 * (A - np.conj(np.transpose(A, (0, 2, 1))))
        T -= np.trace(T, axis1=1, axis2=2)[:, None, None] / 3 * np.eye(3)
        expect = LT.to_complex(f0[mu]) - 2 * T
        got = LT.to_complex(F[mu])
        assert np.max(np.abs(got - expect)) <= 1e-12 * np.max(np.abs(expect))
        G = got - LT.to_complex(f0[mu])
        assert np.max(np.abs(G + np.conj(np.transpose(G, (0, 2, 1))))) <= 1e-12 * np.max(np.abs(G))
        assert np.max(np.abs(np.trace(G, axis1=1, axis2=2))) <= 1e-12 * np.max(np.abs(G))


def _hisq_E(lat, hc, U, eps_naik, midF, midN):
    _, _, W, _ = lat.hisq_links(hc, U, want_W=True)
    ca = hc[5:11]
    cd = (hc[11], 0, 0, 0, 0, hc[12])
    e = 0.0
    for k in range(len(midF)):
        fat, lng = lat.make_imp_links(ca if k == 0 else cd, W, naik=True)
        c = 1.0 if k == 0 else eps_naik[k]
        for mu in range(4):
            e += c * np.sum(np.conj(LT.to_complex(midF[k][mu])) * LT.to_complex(fat[mu])).real
            e += c * np.sum(np.conj(LT.to_complex(midN[k][mu])) * LT.to_complex(lng[mu])).real
    return e


@pytest.mark.parametrize("fat7_lepage", [0, 1])
def test_hisq_deriv_is_the_derivative_of_the_hisq_chain(fat7_lepage):
    """HISQ deriv = dE/dU through asqtad(W) + eps_naik-weighted difference
    terms, the U(3) projection W = V (V^+V)^-1/2 and fat7(U): central finite
    differences of the oracle's own link chain agree to 1e-6."""
    L = (4, 4, 4, 6)
    V = int(np.prod(L))
    lat = O.Lattice(L)
    rng = np.random.default_rng(4)
    hc = LT.hisq_coeff_vector(LT.hisq_bench_coeffs()).copy()
    hc[11], hc[12] = 0.13, -0.21                  # difference one-link, Naik
    hc[13], hc[4] = fat7_lepage, 0.07             # optional fat7 Lepage term
    eps_naik = [0.0, 0.3]
    U = [np.asarray(u) for u in gauge(L, 0.3, 5)]
    midF = [[LT.from_complex(_cgauss(rng, (V, 3, 3))) for _ in range(4)] for _ in range(2)]
    midN = [[LT.from_complex(_cgauss(rng, (V, 3, 3))) for _ in range(4)] for _ in range(2)]
    der = lat.hisq_deriv(hc, U, eps_naik, midF, midN)
    dU = [_cgauss(rng, (V, 3, 3)) for _ in range(4)]
    h = 1e-5
    Up = [LT.from_complex(LT.to_complex(U[m]) + h * dU[m]) for m in range(4)]
    Um = [LT.from_complex(LT.to_complex(U[m]) - h * dU[m]) for m in range(4)]
    fd = (_hisq_E(lat, hc, Up, eps_naik, midF, midN) - _hisq_E(lat, hc, Um, eps_naik, midF, midN)) / (2 * h)
    an = sum(np.sum(np.conj(LT.to_complex(der[m])) * dU[m]).real for m in range(4))
    assert abs(fd - an) <= 1e-6 * abs(an), (fd, an)


def test_hisq_force_groups_and_projection():
    """HISQ force = TA(U (2 deriv)^+) with mids from the sources of each Naik
    group (group 0: all sources; lib/hisq_force_fnmat2_p.c:52-75), residues as
    weights, scale +1 and the sign flip on odd sites."""
    L = (4, 4, 4, 6)
    V = int(np.prod(L))
    lat = O.Lattice(L)
    hc = LT.hisq_coeff_vector(LT.hisq_bench_coeffs()).copy()
    hc[11], hc[12] = 0.13, -0.21
    eps_naik = [0.0, 0.3]
    n_orders = [2, 1]
    U = [np.asarray(u) for u in gauge(L, 0.3, 5)]
    xs = [LT.gaussian_vector(L, 90 + i) for i in range(3)]
    res = [0.5, -0.25, 0.75]
    F = lat.hisq_force(hc, U, eps_naik, res, xs, n_orders)
    sgn = np.where(LT.parity_mask(L), 1.0, -1.0)
    groups = [range(0, 3), range(2, 3)]
    midF, midN = [], []
    for grp in groups:
        gf, gn = [], []
        for mu in range(4):
            mf = np.zeros((V, 3, 3), complex)
            mn = np.zeros((V, 3, 3), complex)
            for i in grp:
                xc = LT.to_complex(xs[i])
                mf += res[i] * np.einsum("va,vb->vab", xc, np.conj(xc[_shift(L, mu, 1)]))
                mn += res[i] * np.einsum("va,vb->vab", xc, np.conj(xc[_shift(L, mu, 3)]))
            gf.append(LT.from_complex(sgn[:, None, None] * mf))
            gn.append(LT.from_complex(sgn[:, None, None] * mn))
        midF.append(gf)
        midN.append(gn)
    der = lat.hisq_deriv(hc, U, eps_naik, midF, midN)
    for mu in range(4):
        A = LT.to_complex(U[mu]) @ np.conj(np.transpose(2 * LT.to_complex(der[mu]), (0, 2, 1)))
        T = 0.5 * (A - np.conj(np.transpose(A, (0, 2, 1))))
        T -= np.trace(T, axis1=1, axis2=2)[:, None, None] / 3 * np.eye(3)
        assert np.max(np.abs(LT.to_complex(F[mu]) - T)) <= 1e-12 * np.max(np.abs(T))


def test_hisq_eps_naik_sets_reduce_to_one_naik():
    """The oracle's n_naiks > 1 link sets (lib/hisq_links_p.c:182-243): fn[0]
    equals the n_naiks = 1 links, fn[k] - fn[0] is eps_k times the difference
    links, and the difference links are the one-link + Naik smearing of W."""
    L = (4, 4, 4, 4)
    lat = O.Lattice(L)
    U = lat.rephase_G(LT.random_gauge(L, 0.5, 9))
    hc = LT.hisq_bench_coeffs()
    hc.difference_one_link, hc.difference_naik = 0.0375, -0.0413
    h = LT.hisq_coeff_vector(hc)
    fat1, lng1, W, _ = lat.hisq_links(h, U, want_W=True)
    sets, (dfat, dlng) = lat.hisq_links_naik(h, U, [0.0, 0.5, -0.25])
    for mu in range(4):
        assert np.array_equal(sets[0][0][mu], fat1[mu]) and np.array_equal(sets[0][1][mu], lng1[mu])
        for k, e in ((1, 0.5), (2, -0.25)):
            assert np.allclose(sets[k][0][mu] - fat1[mu], e * dfat[mu], atol=1e-14)
            assert np.allclose(sets[k][1][mu] - lng1[mu], e * dlng[mu], atol=1e-14)
    # difference links: 0.0375 W (one link only) and -0.0413 W W W (Naik)
    df, dl = lat.make_imp_links([0.0375, 0, 0, 0, 0, -0.0413], W)
    for mu in range(4):
        assert np.array_equal(df[mu], dfat[mu]) and np.array_equal(dl[mu], dlng[mu])
        assert np.allclose(dfat[mu], 0.0375 * np.asarray(W[mu]), atol=1e-14)
