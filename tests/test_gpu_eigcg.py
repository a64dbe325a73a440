"""eigCG (option cg = 1; lib/invert_eigcg_p.c:617-1068, lib/asqtad_invert_p.c:683-770)
through the C ABI: EVENODD solves reach their targets and agree with the
oracle's CG solution; the eigenvalues of the space accumulated in the link
handle converge to the lowest eigenvalues of m^2 - D_eo D_oe (dense
eigen-decomposition of the oracle's operator); later solves start from the
deflated guess and take fewer iterations; a new mass shifts the stored
eigenvalues by the change of m^2; each solve parity keeps its own space."""
import functools

import numpy as np
import pytest

import oracle as O
from conftest import gpu_lattice
from helpers import asqtad_links, full_residual, rel_norm_err
from qopqdp_b200 import lattice as LT
from qopqdp_b200.qop import QOP_EVEN, QOP_ODD, QOP_invert_arg_t, QOP_resid_arg_t

pytestmark = pytest.mark.gpu

L = (4, 4, 4, 8)
V = int(np.prod(L))
VH = V // 2
MASS = 0.02


@functools.lru_cache(maxsize=2)
def dense_low_eigs(mass, eo, n=16):
    """Lowest n eigenvalues of the oracle's m^2 - D_pq D_qp on parity eo."""
    fat, lng = asqtad_links(L, 1.0, 21)
    fo = O.Fla(O.Lattice(L), fat, lng)
    off = 0 if eo == QOP_EVEN else VH
    M = np.zeros((3 * VH, 3 * VH), complex)
    for s in range(VH):
        for c in range(3):
            v = np.zeros((V, 3, 2))
            v[off + s, c, 0] = 1
            o = fo.ddagd(mass, v, eo)[off:off + VH]
            M[:, 3 * s + c] = (o[..., 0] + 1j * o[..., 1]).reshape(-1)
    return np.linalg.eigvalsh(0.5 * (M + M.conj().T))[:n]


def parity_source(seed, eo, dt):
    src = LT.gaussian_vector(L, seed).astype(dt)
    if eo == QOP_EVEN:
        src[VH:] = 0
    else:
        src[:VH] = 0
    return src


def solve(q, fla, fo, mass, src, rsq):
    ia = QOP_invert_arg_t(1e9, 5000, 5000, 5, 2)
    ra = QOP_resid_arg_t(rsq, 0, 0, 0, 0, 0)
    hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
    info = q.invert(fla, mass, hout, hin, ia, ra)
    got = q.extract_V(hout, V).astype(np.float64)
    q.destroy_V(hin)
    q.destroy_V(hout)
    assert info.status == 0
    mq = float(q.real(mass).value)
    return got, ra.final_iter, full_residual(fo, mq, got, src.astype(np.float64))


@pytest.mark.parametrize("prec,rsq,nsolve", [("D", 1e-16, 10), ("F", 1e-10, 8)])
def test_eigcg_converges_to_low_modes(prec, rsq, nsolve):
    q = gpu_lattice(L, prec)
    fat, lng = asqtad_links(L, 1.0, 21)
    dt = q.dtype
    fla = q.create_L_from_raw([a.astype(dt) for a in fat], [a.astype(dt) for a in lng])
    fo = O.Fla(O.Lattice(L), fat, lng)
    assert len(q.eigcg_values(fla, QOP_EVEN)) == 0
    assert q.set_opts(cg=1, eigcg_nev=8, eigcg_m=40, eigcg_l=200) == 0
    try:
        its = []
        for s in range(nsolve):
            src = parity_source(900 + s, QOP_EVEN, dt)
            got, it, true = solve(q, fla, fo, MASS, src, rsq)
            # F3 measures its own residual in single precision; the residual
            # recomputed in double precision sits up to ~100x above the target
            assert true <= rsq * (1.05 if prec == "D" else 200), (s, true)
            if s == 0:
                ref, _ = fo.invert(float(q.real(MASS).value), src.astype(np.float64),
                                   O.InvertArg(1e9, 5000, 5000, 5, 2), O.ResidArg(rsq, 0, 0, 0, 0, 0))
                assert rel_norm_err(got, ref) <= (1e-6 if prec == "D" else 2e-3)
            its.append(it)
        lam = q.eigcg_values(fla, QOP_EVEN)
        exact = dense_low_eigs(MASS, QOP_EVEN)
        print("eigCG iterations", its, "stored", len(lam))
        print("lowest stored", lam[:6], "exact", exact[:6])
        assert len(lam) >= 8 * (nsolve - 1)
        assert np.all(np.diff(lam) >= -1e-12)
        # Rayleigh-Ritz values bound the exact ones from above and the lowest
        # converge first
        tol = 1e-6 if prec == "D" else 1e-3
        assert np.all(lam[:4] >= exact[:4] * (1 - tol))
        assert np.allclose(lam[:4], exact[:4], rtol=1e-4 if prec == "D" else 5e-3, atol=0)
        assert np.mean(its[-3:]) <= 0.92 * its[0], its
        assert len(q.eigcg_values(fla, QOP_ODD)) == 0
    finally:
        assert q.set_opts(cg=0) == 0
        q.destroy_L(fla)


def test_eigcg_mass_shift_and_parities():
    q = gpu_lattice(L, "D")
    fat, lng = asqtad_links(L, 1.0, 21)
    fla = q.create_L_from_raw(fat, lng)
    fo = O.Fla(O.Lattice(L), fat, lng)
    assert q.set_opts(cg=1, eigcg_nev=8, eigcg_m=40, eigcg_l=200) == 0
    try:
        for s in range(6):
            solve(q, fla, fo, MASS, parity_source(950 + s, QOP_EVEN, np.float64), 1e-16)
        lam0 = q.eigcg_values(fla, QOP_EVEN)
        # a heavier mass: the stored space is reused with l + (m'^2 - m^2)
        m2 = 0.05
        got, it, true = solve(q, fla, fo, m2, parity_source(960, QOP_EVEN, np.float64), 1e-16)
        assert true <= 1.05e-16
        lam1 = q.eigcg_values(fla, QOP_EVEN)
        assert len(lam1) >= len(lam0)
        # (the end-of-solve Rayleigh-Ritz step refines the shifted values)
        assert abs(lam1[0] - (lam0[0] + m2 * m2 - MASS * MASS)) <= 1e-4 * lam1[0]
        exact = dense_low_eigs(m2, QOP_EVEN, 4)
        assert np.allclose(lam1[:2], exact[:2], rtol=1e-5, atol=0)
        # an odd-parity source builds a separate space and leaves the even one
        n_even = len(lam1)
        got, it, true = solve(q, fla, fo, MASS, parity_source(970, QOP_ODD, np.float64), 1e-16)
        assert true <= 1.05e-16
        assert len(q.eigcg_values(fla, QOP_ODD)) >= 8
        assert len(q.eigcg_values(fla, QOP_EVEN)) == n_even
        # sources on both parities: the solve parity follows the larger half
        got, it, true = solve(q, fla, fo, MASS, LT.gaussian_vector(L, 980), 1e-16)
        assert true <= 1.05e-16
    finally:
        assert q.set_opts(cg=0) == 0
        q.destroy_L(fla)


def test_eigcg_options_and_errors():
    q = gpu_lattice(L, "D")
    fat, lng = asqtad_links(L, 1.0, 21)
    fla = q.create_L_from_raw(fat, lng)
    # window too small for 2 nev + 2: the solve reports failure, nothing runs
    assert q.set_opts(cg=1, eigcg_nev=8, eigcg_m=10, eigcg_l=64) == 0
    src = LT.gaussian_vector(L, 850)
    hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
    info = q.invert(fla, 0.05, hout, hin, QOP_invert_arg_t(1e9, 1000, 1000, 5, 2),
                    QOP_resid_arg_t(1e-16, 0, 0, 0, 0, 0))
    assert info.status != 0
    assert q.set_opts(cg=0, eigcg_nev=10, eigcg_m=100, eigcg_l=200) == 0
    with pytest.raises(RuntimeError):
        q.eigcg_values(fla, 2)   # QOP_EVENODD has no space
    q.destroy_V(hin)
    q.destroy_V(hout)
    q.destroy_L(fla)
