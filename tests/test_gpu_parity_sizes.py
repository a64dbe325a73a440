"""Parity at the workloads' own sizes, through the C ABI.

* Config 1 (asqtad F3 and D3, 8^4, eps 0.3, m 0.1): all nine
  (eo_out, eo_in) cases of QOP_*_asqtad_dslash (lib/asqtad_dslash_p.c:1048-1092)
  against the FP64 oracle, D3 <= 1e-13 and F3 <= 2e-6 relative per site.
* 24^4 (165,888 sites per parity, 1,296 site blocks of 128: the persistent
  int16 hop grid of 148 x 5 blocks strides over them twice): the nine cases
  again, and the int16 sloppy operator of the mixed solvers (the default
  packed persistent hop, the fused-update second hop, and the other hop
  shapes) compared site by site with the FP64 operator applied to exactly the
  values the device stores (tests/q16ref.py), with the bound stated there:
  |got - ref| <= 4e-5 |ref| + 1e-6 sum_k |U_k| |v_k| per site.  The norm-wise
  distance to the unquantised FP64 operator is checked too (<= 2^-12).
* The 16-system batched hop (default 8 systems per thread) and the 12-system
  shape (4 per thread) on the same lattice, system by system, and the
  tensor-core hop (batch_kernel 16: mma.sync on bf16 hi / lo operands) with
  16, 12 and 3 systems against the same FP64 operator on its own storage.
"""
import itertools

import numpy as np
import pytest

import oracle as O
import q16ref as R
from conftest import gpu_lattice
from helpers import asqtad_links, hisq_links, site_rel_err
from qopqdp_b200 import lattice as LT

pytestmark = pytest.mark.gpu

TOL = {"D": 1e-13, "F": 2e-6}
COMBOS = list(itertools.product([0, 1, 2], [0, 1, 2]))
BIG = (24, 24, 24, 24)


def _nine_cases(L, prec, kind="asqtad"):
    q = gpu_lattice(L, prec)
    if kind == "asqtad":
        fat, lng = asqtad_links(L, 0.3, 7)
    else:
        fat, lng, _, _ = hisq_links(L, 0.5, 9)
    dt = np.float32 if prec == "F" else np.float64
    fat = [np.asarray(a, dtype=dt) for a in fat]
    lng = [np.asarray(a, dtype=dt) for a in lng]
    fo = O.Fla(O.Lattice(L), [a.astype(np.float64) for a in fat], [a.astype(np.float64) for a in lng])
    fla = q.create_L_from_raw(fat, lng)
    V = int(np.prod(L))
    src = LT.gaussian_vector(L, 3).astype(dt)
    worst = 0.0
    for eo_out, eo_in in COMBOS:
        init = LT.gaussian_vector(L, 4).astype(dt)
        hin, hout = q.create_V(src), q.create_V(init)
        q.dslash(fla, 0.1, hout, hin, eo_out, eo_in)
        got = q.extract_V(hout, V)
        ref = fo.dslash(float(q.real(0.1).value), src.astype(np.float64), eo_out, eo_in,
                        out=init.astype(np.float64))
        err = site_rel_err(got, ref)
        worst = max(worst, err)
        assert err <= TOL[prec], (L, prec, eo_out, eo_in, err)
        q.destroy_V(hin)
        q.destroy_V(hout)
    q.destroy_L(fla)
    print("nine cases %s %s: worst site error %.2e" % (L, prec, worst))


@pytest.mark.parametrize("prec", ["F", "D"])
def test_config1_dslash_nine_cases_8x8x8x8(prec):
    _nine_cases((8, 8, 8, 8), prec)


@pytest.mark.parametrize("prec", ["D", "F"])
def test_dslash_nine_cases_24x24x24x24_hisq(prec):
    _nine_cases(BIG, prec, kind="hisq")


@pytest.fixture(scope="module")
def big_hisq():
    fat, lng, _, _ = hisq_links(BIG, 0.5, 9)
    geo = R.Geometry(BIG)
    dbl = R.dbl_links(geo, fat, lng)
    dq, recon = R.quantize_links(dbl)
    return fat, lng, geo, dbl, dq, recon


# per-site bounds (tests/q16ref.py site_err): int16 vectors round the output
# to 15 bits of the site's largest component; the tensor-core form stores
# bf16 hi + lo (16 bits of each component) and represents the int16 links as
# bf16 hi + lo too (2^-17 of each element) and drops lo . lo (2^-18 of each
# product), so its arithmetic term is larger and its output term smaller
BOUNDS = {"q16": dict(out_scale=4e-5, acc_scale=1e-6), "b16": dict(out_scale=1e-5, acc_scale=1.5e-5)}


def _check_sloppy(geo, dbl, dq, mass, src, t_got, a_got, eo, label, fmt="q16"):
    V = geo.V
    q_, p_ = 1 - eo, eo
    sq, sp = R.parity_sites(V, q_), R.parity_sites(V, p_)
    p = np.zeros((V, 3), complex)
    p[sp] = (R.quantize_vector if fmt == "q16" else R.split_vector)(R.cplx(src)[sp])
    # first hop on exactly the stored p and links
    t_ref, t_mag = R.hop(geo, dq, p, sq)
    e1 = R.site_err(R.cplx(t_got)[sq], t_ref, t_mag, **BOUNDS[fmt])
    # second hop on exactly the stored t (the device's own output)
    t = np.zeros((V, 3), complex)
    t[sq] = R.cplx(t_got)[sq]
    h2, m2mag = R.hop(geo, dq, t, sp)
    a_ref = mass * mass * p[sp] - h2
    e2 = R.site_err(R.cplx(a_got)[sp], a_ref, m2mag + mass * mass * np.sqrt((np.abs(p[sp]) ** 2).sum(axis=1)),
                    **BOUNDS[fmt])
    # distance to the unquantised FP64 operator
    x = np.zeros((V, 3), complex)
    x[sp] = R.cplx(src)[sp]
    tx, _ = R.hop(geo, dbl, x, sq)
    tt = np.zeros((V, 3), complex)
    tt[sq] = tx
    hx, _ = R.hop(geo, dbl, tt, sp)
    ax = mass * mass * x[sp] - hx
    d = float(np.linalg.norm(R.cplx(a_got)[sp] - ax) / np.linalg.norm(ax))
    print("%s: t %.3f, Ap %.3f of the bound; |Ap - A x| / |A x| = %.2e" % (label, e1, e2, d))
    assert e1 <= 1.0 and e2 <= 1.0, (label, e1, e2)
    assert d <= 2.0 ** -12, (label, d)
    return t, p


@pytest.mark.parametrize("variant,kind2", [(25, 3), (25, 2), (15, 2), (0, 2)])
def test_int16_operator_matches_fp64_per_site_24x24x24x24(big_hisq, variant, kind2):
    fat, lng, geo, dbl, dq, recon = big_hisq
    assert recon, "HISQ Naik links are |c| x unitary: the device rebuilds row 2"
    q = gpu_lattice(BIG, "D")
    V = geo.V
    fla = q.create_L_from_raw(fat, lng)
    mass = 0.01
    for eo in (0, 1):
        src = LT.gaussian_vector(BIG, 40 + eo)
        hin = q.create_V(src)
        ht, ha = q.create_V(np.zeros_like(src)), q.create_V(np.zeros_like(src))
        st, sums = q.sloppy_ddagd(fla, mass, ht, ha, hin, eo, variant, kind2)
        assert st == 0
        t_got, a_got = q.extract_V(ht, V), q.extract_V(ha, V)
        t, p = _check_sloppy(geo, dbl, dq, mass, src, t_got, a_got, eo, "variant %d kind %d eo %d" % (variant, kind2, eo))
        # the reductions are those of the stored vectors (a site left out or
        # counted twice would move them by ~1e-5)
        sp = R.parity_sites(V, eo)
        ap = R.cplx(a_got)[sp]
        n2 = lambda z: float((z.real ** 2 + z.imag ** 2).sum())
        ref = [n2(t), n2(p), float(np.vdot(p[sp], ap).real), n2(ap)]
        rel = [abs(a - b) / abs(b) for a, b in zip(sums, ref)]
        print("reductions vs the stored vectors: %s" % " ".join("%.1e" % r for r in rel[: 4 if kind2 == 3 else 2]))
        assert rel[0] <= 1e-9 and rel[1] <= 1e-9
        if kind2 == 3:
            assert rel[2] <= 1e-9 and rel[3] <= 1e-9
        for h in (hin, ht, ha):
            q.destroy_V(h)
    q.destroy_L(fla)


@pytest.mark.parametrize("n,variant", [(16, -1), (12, -1), (16, 12), (16, 16), (12, 16), (3, 16)])
def test_batched_int16_operator_matches_fp64_per_site_24x24x24x24(big_hisq, n, variant):
    fat, lng, geo, dbl, dq, recon = big_hisq
    q = gpu_lattice(BIG, "D")
    V = geo.V
    fla = q.create_L_from_raw(fat, lng)
    eo = 0
    masses = [0.01 * (1.5 ** j) for j in range(n)]
    srcs = [LT.gaussian_vector(BIG, 100 + j) for j in range(n)]
    hin = [q.create_V(s) for s in srcs]
    ht = [q.create_V(np.zeros_like(srcs[0])) for _ in range(n)]
    ha = [q.create_V(np.zeros_like(srcs[0])) for _ in range(n)]
    st, sums = q.sloppy_ddagd_batch(fla, masses, ht, ha, hin, eo, variant)
    assert st == 0
    fmt = "b16" if variant == 16 else "q16"
    for j in sorted({0, n // 2, n - 1}):      # first, middle and last system of the launch
        t, p = _check_sloppy(geo, dbl, dq, masses[j], srcs[j], q.extract_V(ht[j], V), q.extract_V(ha[j], V), eo,
                             "batch n %d variant %d system %d" % (n, variant, j), fmt)
        t2 = (np.abs(t) ** 2).sum()
        # the batched hops reduce |t|^2 before rounding t to its storage
        assert abs(sums[j][0] - t2) <= 1e-4 * t2
        pap = t2 + masses[j] ** 2 * (np.abs(p) ** 2).sum()
        assert abs(sums[j][1] - pap) <= 1e-4 * pap
    for h in hin + ht + ha:
        q.destroy_V(h)
    q.destroy_L(fla)


def test_config3_multimass_every_mass_meets_target():
    """Config 3 at its own size: HISQ 24^3x48 (eps 0.5, links built on the
    device), one source, 12 masses sqrt(logspace(-4, 0)), rsqmin 1e-20,
    through QOP_D3_asqtad_invert_multi with the int16 defaults (multi-shift
    phase, then the batched refinement).  Every mass's solution, checked by
    the oracle's FP64 operator on the device's own links
    (examples/asqtad_test.c:84-130 check_resids), has
    |b - A x|^2 / |b|^2 <= 1.05e-20, and the reported final_rsq is that
    true residual."""
    from qopqdp_b200.qop import QOP_invert_arg_t, QOP_resid_arg_t, QOP_EVEN
    from helpers import eo_residual
    L = (24, 24, 24, 48)
    V = int(np.prod(L))
    q = gpu_lattice(L, "D")
    G = q.create_G(LT.random_gauge(L, 0.5, 2024, device="cuda"))
    q.rephase_G(G, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
    H = q.hisq_create_L_from_G(LT.hisq_bench_coeffs(), G)
    fla = q.hisq_asqtad_links(H, 0)
    q.destroy_G(G)
    masses = [float(x) for x in np.sqrt(np.logspace(-4, 0, 12))]
    src = LT.gaussian_vector(L, 2024)
    hin = q.create_V(src, QOP_EVEN)
    outs = [q.create_V(np.zeros_like(src)) for _ in masses]
    ras = [QOP_resid_arg_t(1e-20, 0, 0, 0, 0, 0) for _ in masses]
    assert q.set_opts(prec_sloppy=16) == 0
    try:
        info = q.invert_multi(fla, [masses], [outs], [hin], QOP_invert_arg_t(1e9, 200000, 200000, 50, QOP_EVEN),
                              [ras])
    finally:
        assert q.set_opts(prec_sloppy=64) == 0
    assert info.status == 0
    fat, lng = q.extract_L(fla, V)
    fo = O.Fla(O.Lattice(L), fat, lng)
    for k, m in enumerate(masses):
        x = q.extract_V(outs[k], V)
        true = eo_residual(fo, m, x, src, L, 0)
        assert true <= 1.05e-20, (m, true)
        assert abs(ras[k].final_rsq - true) <= 0.05 * true + 1e-26, (m, ras[k].final_rsq, true)
        q.destroy_V(outs[k])
    q.destroy_V(hin)
    q.hisq_destroy_L(H)
