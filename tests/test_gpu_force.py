"""Asqtad fermion force through the C ABI (QOP_*_asqtad_force_multi,
lib/asqtad_force_p.c:16-64) against the oracle on identical inputs: the
outer products of the sources, the derivative through the smeared links
(one-link, 3-, 5-, 7-staple, Lepage and Naik terms) and the traceless
anti-Hermitian projection, accumulated into an existing force field."""
import numpy as np
import pytest

import oracle as O
from conftest import gpu_lattice
from helpers import gauge
from qopqdp_b200 import lattice as LT
from qopqdp_b200.qop import QOP_info_t

pytestmark = pytest.mark.gpu

L = (4, 4, 4, 8)
V = int(np.prod(L))


def _run(prec, coef, nsrc):
    q = gpu_lattice(L, prec)
    U = [np.asarray(u) for u in gauge(L, 0.3, 5)]
    xs = [LT.gaussian_vector(L, 80 + i) for i in range(nsrc)]
    eps = [0.7, -0.4, 0.25][:nsrc]
    rng = np.random.default_rng(2)
    f0 = [rng.standard_normal((V, 3, 3, 2)) * 0.1 for _ in range(4)]
    ref = O.Lattice(L).asqtad_force(coef, U, eps, xs, force=f0)
    dt = q.dtype
    G = q.create_G([u.astype(dt) for u in U])
    F = q.create_F([f.astype(dt) for f in f0])
    hv = [q.create_V(x.astype(dt)) for x in xs]
    info = q.asqtad_force(G, F, coef, eps, hv)
    got = q.extract_F(F, V)
    for h in hv:
        q.destroy_V(h)
    q.destroy_F(F)
    q.destroy_G(G)
    return info, got, ref, f0


@pytest.mark.parametrize("coef", [(1.0, 0.1, 0.1, 0.1, 0.1, 0.1), (0.7, -0.23, 0.31, -0.17, 0.29, -0.13),
                                  (1.0, 0.2, 0.0, 0.0, 0.0, 0.0)])
@pytest.mark.parametrize("nsrc", [1, 3])
def test_force_matches_oracle_d3(coef, nsrc):
    info, got, ref, f0 = _run("D", coef, nsrc)
    assert info.status == 0
    scale = max(np.max(np.abs(r - f)) for r, f in zip(ref, f0))
    for g_, r in zip(got, ref):
        assert np.max(np.abs(g_ - r)) <= 1e-12 * scale


def test_force_matches_oracle_f3():
    info, got, ref, f0 = _run("F", (1.0, 0.1, 0.1, 0.1, 0.1, 0.1), 2)
    assert info.status == 0
    scale = max(np.max(np.abs(r - f)) for r, f in zip(ref, f0))
    for g_, r in zip(got, ref):
        assert np.max(np.abs(g_.astype(np.float64) - r)) <= 2e-5 * scale


def test_force_errors_and_options():
    q = gpu_lattice(L, "D")
    U = [np.asarray(u) for u in gauge(L, 0.3, 5)]
    G = q.create_G(U)
    F = q.create_F([np.zeros((V, 3, 3, 2)) for _ in range(4)])
    hv = q.create_V(LT.gaussian_vector(L, 90))
    info = q.asqtad_force(G, None, (1, 0.1, 0.1, 0.1, 0.1, 0.1), [0.5], [hv])
    assert info.status != 0                                   # NULL force handle
    info = q.asqtad_force(G, F, (1, 0.1, 0.1, 0.1, 0.1, 0.1), [0.5], [None])
    assert info.status != 0                                   # NULL source
    from qopqdp_b200.qop import _c_opts
    arr, _k = _c_opts({"fnmat_src_min": 1, "veclength": 8})
    assert q.lib.QOP_asqtad_force_set_opts(arr, 2) == 0
    arr, _k = _c_opts({"veclength": 0})
    assert q.lib.QOP_asqtad_force_set_opts(arr, 1) != 0
    arr, _k = _c_opts({"fnmat_src_min": 2, "veclength": 4})   # the defaults again
    assert q.lib.QOP_asqtad_force_set_opts(arr, 2) == 0
    q.destroy_V(hv)
    q.destroy_F(F)
    q.destroy_G(G)


@pytest.mark.parametrize("prec,tol", [("D", 1e-10), ("F", 5e-5)])
def test_hisq_force_matches_oracle(prec, tol):
    """QOP_*_hisq_force_multi (lib/hisq_force_p.c:50-80) with two Naik
    epsilon groups: asqtad level on W, difference terms weighted by
    eps_naik, the U(3) projection adjoint and the fat7 level, against the
    oracle on the same gauge field and sources."""
    q = gpu_lattice(L, prec)
    hc = LT.hisq_bench_coeffs()
    hc.n_naiks = 2
    hc.eps_naik[1] = 0.3
    hc.difference_one_link, hc.difference_naik = 0.13, -0.21
    U = [np.asarray(u) for u in gauge(L, 0.3, 5)]
    xs = [LT.gaussian_vector(L, 95 + i) for i in range(3)]
    res, n_orders = [0.5, -0.25, 0.75], [2, 1]
    rng = np.random.default_rng(6)
    f0 = [rng.standard_normal((V, 3, 3, 2)) * 0.1 for _ in range(4)]
    ref = O.Lattice(L).hisq_force(LT.hisq_coeff_vector(hc), U, [0.0, 0.3], res, xs, n_orders, force=f0)
    dt = q.dtype
    q.set_hisq_opts(want_aux=1)
    G = q.create_G([u.astype(dt) for u in U])
    H = q.hisq_create_L_from_G(hc, G)
    F = q.create_F([f.astype(dt) for f in f0])
    hv = [q.create_V(x.astype(dt)) for x in xs]
    info = q.hisq_force(H, F, hc, res, hv, n_orders)
    got = q.extract_F(F, V)
    assert info.status == 0
    scale = max(np.max(np.abs(r - f)) for r, f in zip(ref, f0))
    for g_, r in zip(got, ref):
        assert np.max(np.abs(g_.astype(np.float64) - r)) <= tol * scale
    # without the auxiliary fields the force is refused
    q.set_hisq_opts(want_aux=0)
    H2 = q.hisq_create_L_from_G(hc, G)
    assert q.hisq_force(H2, F, hc, res, hv, n_orders).status != 0
    q.set_hisq_opts(want_aux=1)
    for h in hv:
        q.destroy_V(h)
    q.hisq_destroy_L(H)
    q.hisq_destroy_L(H2)
    q.destroy_F(F)
    q.destroy_G(G)


@pytest.mark.parametrize("nsrc,fsm", [(1, 0), (1, 2), (3, 2), (3, 4)])
def test_force_algorithm_choice_matches_oracle(nsrc, fsm):
    """The reference picks ASVEC for nsrc < fnmat_src_min and FNMAT otherwise
    (lib/asqtad_force_p.c:22-37); compiled from its sources, ASVEC stores
    TA(force + C) with TA(C) half the FNMAT term.  The device follows the
    option like the reference, checked against the oracle with the same
    choice (accumulating into a force field that is not anti-Hermitian, so
    the ASVEC projection of the incoming force shows)."""
    from qopqdp_b200.qop import _c_opts
    q = gpu_lattice(L, "D")
    U = [np.asarray(u) for u in gauge(L, 0.3, 5)]
    xs = [LT.gaussian_vector(L, 80 + i) for i in range(nsrc)]
    eps = [0.7, -0.4, 0.25][:nsrc]
    coef = (1.0, 0.1, 0.1, 0.1, 0.1, 0.1)
    f0 = [np.random.default_rng(3).standard_normal((V, 3, 3, 2)) * 0.1 for _ in range(4)]
    ref = O.Lattice(L).asqtad_force(coef, U, eps, xs, force=f0, fnmat_src_min=fsm)
    arr, _k = _c_opts({"fnmat_src_min": fsm})
    assert q.lib.QOP_asqtad_force_set_opts(arr, 1) == 0
    try:
        G = q.create_G(U)
        F = q.create_F(f0)
        hv = [q.create_V(x) for x in xs]
        assert q.asqtad_force(G, F, coef, eps, hv).status == 0
        got = q.extract_F(F, V)
    finally:
        arr, _k = _c_opts({"fnmat_src_min": 2})
        assert q.lib.QOP_asqtad_force_set_opts(arr, 1) == 0
    scale = max(np.max(np.abs(r)) for r in ref)
    for g_, r in zip(got, ref):
        assert np.max(np.abs(g_ - r)) <= 1e-12 * scale
    for h in hv:
        q.destroy_V(h)
    q.destroy_F(F)
    q.destroy_G(G)
