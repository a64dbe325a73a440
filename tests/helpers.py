"""Shared test fixtures: seeded inputs, oracle operators, error metrics."""
import functools

import numpy as np

import oracle as O
from qopqdp_b200 import lattice as LT


@functools.lru_cache(maxsize=8)
def gauge(L, eps, seed, phases=True):
    U = LT.random_gauge(L, eps, seed)
    if phases:
        U = O.Lattice(L).rephase_G(U, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
    return tuple(np.ascontiguousarray(u) for u in U)


@functools.lru_cache(maxsize=8)
def asqtad_links(L, eps, seed, naik=True):
    lat = O.Lattice(L)
    fat, lng = lat.make_imp_links(LT.ASQTAD_BENCH_COEFFS, list(gauge(L, eps, seed)), naik=naik)
    return tuple(fat), (tuple(lng) if lng is not None else None)


@functools.lru_cache(maxsize=4)
def hisq_links(L, eps, seed):
    lat = O.Lattice(L)
    hc = LT.hisq_coeff_vector(LT.hisq_bench_coeffs())
    fat, lng, W, n = lat.hisq_links(hc, list(gauge(L, eps, seed)), want_W=True)
    return tuple(fat), tuple(lng), tuple(W), n


def site_rel_err(a, ref):
    """max over sites of |a(x)-ref(x)| / |ref(x)| (3-colour complex norms)."""
    a = np.asarray(a, dtype=np.float64).reshape(a.shape[0], -1)
    ref = np.asarray(ref, dtype=np.float64).reshape(ref.shape[0], -1)
    num = np.sqrt(((a - ref) ** 2).sum(axis=1))
    den = np.sqrt((ref ** 2).sum(axis=1))
    mask = den > 0
    if not mask.any():
        return float(num.max())
    out = (num[mask] / den[mask]).max()
    if (~mask).any():
        out = max(out, float(num[~mask].max()))
    return float(out)


def rel_norm_err(a, ref):
    a = np.asarray(a, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    return float(np.sqrt(((a - ref) ** 2).sum() / max((ref ** 2).sum(), 1e-300)))


def half(a, L, eo):
    V = int(np.prod(L))
    if eo == 0:
        return a[: V // 2]
    if eo == 1:
        return a[V // 2:]
    return a


def eo_residual(fla_oracle, m, out, src, L, eo):
    """examples/asqtad_test.c:84-130 check_resids: |in - (1/m)(m^2 - D D) out|^2/|in|^2 on eo."""
    t = fla_oracle.dslash(m, out, O.EVENODD, eo)
    chk = fla_oracle.dslash(-m, t, eo, O.EVENODD)
    r = half(chk, L, eo) / m + half(src, L, eo)
    return float((r ** 2).sum() / (half(src, L, eo) ** 2).sum())


def full_residual(fla_oracle, m, out, src):
    Dx = fla_oracle.dslash(m, out, O.EVENODD, O.EVENODD)
    return float(((Dx - src) ** 2).sum() / (src ** 2).sum())
