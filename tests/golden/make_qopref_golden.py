"""Writes tests/golden/qopref_4x4x4x4.npz: outputs of the reference's own
asqtad/HISQ path (QOPQDP 0.21.1, compiled unmodified from its sources by
oracle/ref into oracle/_ref/libqopref.so) on seeded inputs, so that the
oracle and the GPU path can be checked against the reference where its
sources are absent.

Inputs are regenerated from seeds by qopqdp_b200.lattice (the file keeps a
checksum of each, to catch a generator change):
  gauge      random_gauge((4,4,4,4), eps=0.3, seed=7), rephased by the
             reference's QOP_rephase_G_qdp (r0 = 0, t antiperiodic, staggered
             sign masks 0,1,3,7: examples/asqtad_test.c:275-281)
  source     gaussian_vector(L, 41) (V x 3 complex)
Outputs (reference D3 build):
  asq_*      asqtad links (coefficients 1, .1, .1, .1, .1, .1) of
             QOP_asqtad_create_L_from_G; Dslash EVENODD<-EVENODD and
             EVEN<-ODD at mass 0.1; EVEN solve (m A^-1 b, rsqmin 1e-20);
             invert_multi on ODD with masses 0.1, 0.2, 0.4 (rsqmin 1e-20)
  hisq_*     HISQ links (examples/hisq_invert_bench.c coefficients, U(3),
             analytic projection) of QOP_hisq_create_L_from_G; Dslash
             EVENODD<-EVENODD at mass 0.05
  force_*    fermion forces on a rough field, random_gauge(L, 0.5, seed=2)
             rephased as above (two fat7 links with a V^+V eigenvalue below
             the 5e-5 force filter), sources gaussian_vector(L, 51 + i):
             force_asq_asvec  QOP_asqtad_force_multi, one source, eps 0.3
                              (ASVEC: below fnmat_src_min = 2)
             force_asq_fnmat  the same with three sources, eps .3 -.2 .5
             force_hisq       QOP_hisq_force_multi, three sources, residues
                              .3 -.2 .5, Naik groups [2, 1] with eps_naik
                              (0, 0.1), difference one-link .3 / Naik -.05,
                              default force filter
  *_ck       link checksums: sum of squares and sum of w * links with the
             fixed weights w = cos(0.37 k) over the flattened array
Run from the repository root: python tests/golden/make_qopref_golden.py
(it builds oracle/_ref first when the reference sources are present).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import refqop as R  # noqa: E402
from oracle import InvertArg, ResidArg  # noqa: E402
from qopqdp_b200 import lattice as LT  # noqa: E402

L = (4, 4, 4, 4)
V = 256
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "qopref_4x4x4x4.npz")


def checksum(arrs):
    a = np.concatenate([np.asarray(x, dtype=np.float64).ravel() for x in arrs])
    w = np.cos(0.37 * np.arange(a.size))
    return np.array([float((a * a).sum()), float((a * w).sum())])


def main():
    R.build()
    U = LT.random_gauge(L, 0.3, 7)
    G = R.rephase_G(L, U, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
    src = LT.gaussian_vector(L, 41).reshape(V, 6)
    out = {"L": np.array(L), "gauge_ck": checksum(U), "src_ck": checksum([src]), "rephased_ck": checksum(G)}

    fat, lng = R.asqtad_links(L, LT.ASQTAD_BENCH_COEFFS, G)
    out["asq_fat_ck"], out["asq_long_ck"] = checksum(fat), checksum(lng)
    fla = R.RefFla(L, fat, lng, R.D3)
    out["asq_dslash_eoeo"] = fla.dslash(0.1, src, 2, 2)
    out["asq_dslash_e_o"] = fla.dslash(0.1, src, 0, 1)
    ra = ResidArg(1e-20, 0, 0, 0, 0, 0)
    x, _ = fla.invert(0.1, src, InvertArg(1e9, 2000, 1000, 5, 0), ra)
    out["asq_invert_even"] = x[: V // 2]
    out["asq_invert_even_iters"] = np.array([ra.final_iter, ra.final_restart])
    masses = [0.1, 0.2, 0.4]
    ras = [[ResidArg(1e-20, 0, 0, 0, 0, 0) for _ in masses]]
    xs, _ = fla.invert_multi([masses], [src], InvertArg(1e9, 2000, 1000, 5, 1), ras)
    out["asq_multi_odd"] = np.stack([x[V // 2:] for x in xs[0]])
    out["asq_multi_odd_iters"] = np.array([r.final_iter for r in ras[0]])

    hc = LT.hisq_coeff_vector(LT.hisq_bench_coeffs())
    sets, W, _ = R.hisq_links(L, hc, G)
    hfat, hlng = sets[0]
    out["hisq_fat_ck"], out["hisq_long_ck"], out["hisq_W_ck"] = checksum(hfat), checksum(hlng), checksum(W)
    hfla = R.RefFla(L, hfat, hlng, R.D3)
    out["hisq_dslash_eoeo"] = hfla.dslash(0.05, src, 2, 2)

    Ur = LT.random_gauge(L, 0.5, 2)
    Gr = R.rephase_G(L, Ur, LT.BENCH_R0, LT.BENCH_BC, LT.BENCH_SIGNMASK)
    out["force_gauge_ck"] = checksum(Ur)
    xs = [LT.gaussian_vector(L, 51 + i).reshape(V, 6) for i in range(3)]
    eps = [0.3, -0.2, 0.5]
    out["force_asq_asvec"] = np.stack(R.asqtad_force(L, LT.ASQTAD_BENCH_COEFFS, Gr, eps[:1], xs[:1]))
    out["force_asq_fnmat"] = np.stack(R.asqtad_force(L, LT.ASQTAD_BENCH_COEFFS, Gr, eps, xs))
    hf = LT.hisq_coeff_vector(LT.hisq_bench_coeffs())
    hf[11], hf[12] = 0.3, -0.05
    out["force_hisq"] = np.stack(R.hisq_force(L, hf, Gr, [0.0, 0.1], eps, xs, [2, 1]))
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
