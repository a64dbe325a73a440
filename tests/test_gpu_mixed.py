"""Mixed-precision reliable-update solves (prec_sloppy 16 / 32) reach the
requested FP64 true residual and agree with the FP64 oracle solve within
the accuracy the tolerance implies."""
import numpy as np
import pytest

import oracle as O
from conftest import gpu_lattice
from helpers import hisq_links, asqtad_links, eo_residual, rel_norm_err, half
from qopqdp_b200 import lattice as LT
from qopqdp_b200.qop import QOP_invert_arg_t, QOP_resid_arg_t

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [16, 32])
@pytest.mark.parametrize("L,kind,m", [((4, 4, 4, 8), "hisq", 0.05), ((8, 8, 8, 8), "asqtad", 0.02)])
def test_mixed_solve_reaches_fp64_tolerance(prec, L, kind, m):
    q = gpu_lattice(L, "D")
    V = int(np.prod(L))
    if kind == "hisq":
        fat, lng, _, _ = hisq_links(L, 0.5, 9)
    else:
        fat, lng = asqtad_links(L, 0.3, 7)
    fo = O.Fla(O.Lattice(L), fat, lng)
    fla = q.create_L_from_raw(fat, lng)
    src = LT.gaussian_vector(L, 101)
    for eo in (0, 1):
        for rsq in (1e-20, 1e-14):
            assert q.set_opts(prec_sloppy=prec) == 0
            ia = QOP_invert_arg_t(1e9, 20000, 20000, 5, eo)
            ra = QOP_resid_arg_t(rsq, 0, 0, 0, 0, 0)
            hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
            q.invert(fla, m, hout, hin, ia, ra)
            got = q.extract_V(hout, V)
            true = eo_residual(fo, m, got, src, L, eo)
            assert true <= rsq * 1.05, (prec, eo, rsq, true, ra.final_iter)
            assert abs(ra.final_rsq - true) <= 0.05 * true + 1e-26
            assert ra.final_iter > 0 and ra.final_restart <= 1
            # same system solved by the FP64 oracle: solutions agree to the
            # accuracy the residual allows (condition number ~ 1/m^2)
            oia, ora = O.InvertArg(1e9, 20000, 20000, 5, eo), O.ResidArg(rsq, 0, 0, 0, 0, 0)
            ref, _ = fo.invert(m, src, oia, ora)
            assert rel_norm_err(half(got, L, eo), half(ref, L, eo)) <= max(1e-6, 30 * np.sqrt(rsq) / m ** 2)
            q.destroy_V(hin)
            q.destroy_V(hout)
    assert q.set_opts(prec_sloppy=64) == 0
    q.destroy_L(fla)


def test_mixed_iterations_close_to_fp64():
    """FP16 storage costs a bounded number of extra iterations."""
    L = (8, 8, 8, 8)
    q = gpu_lattice(L, "D")
    fat, lng = asqtad_links(L, 0.3, 7)
    fla = q.create_L_from_raw(fat, lng)
    src = LT.gaussian_vector(L, 102)
    its = {}
    for prec in (64, 32, 16):
        q.set_opts(prec_sloppy=prec)
        ia = QOP_invert_arg_t(1e9, 20000, 20000, 5, 0)
        ra = QOP_resid_arg_t(1e-20, 0, 0, 0, 0, 0)
        hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
        q.invert(fla, 0.02, hout, hin, ia, ra)
        its[prec] = ra.final_iter
        assert ra.final_rsq <= 1.05e-20
        q.destroy_V(hin)
        q.destroy_V(hout)
    q.set_opts(prec_sloppy=64)
    assert its[32] <= 1.3 * its[64] + 20 and its[16] <= 2.0 * its[64] + 50, its
    q.destroy_L(fla)


@pytest.mark.parametrize("kind", ["hisq", "random_long"])
def test_long_link_reconstruction(kind):
    """int16 long links stored as two rows + det phase (when they are |c| times
    a unitary matrix) give the same convergence as full storage; links that
    are not of that form fall back to full storage automatically."""
    L = (4, 4, 4, 8)
    V = int(np.prod(L))
    q = gpu_lattice(L, "D")
    fat, lng, _, _ = hisq_links(L, 0.5, 9)
    if kind == "random_long":
        rng = np.random.default_rng(5)
        lng = tuple(0.05 * rng.standard_normal(a.shape) for a in lng)
    fo = O.Fla(O.Lattice(L), fat, lng)
    fla = q.create_L_from_raw(fat, lng)
    src = LT.gaussian_vector(L, 300)
    its = {}
    for recon in (1, 0):
        assert q.set_opts(prec_sloppy=16, recon_long=recon) == 0
        ia = QOP_invert_arg_t(1e9, 20000, 20000, 5, 0)
        ra = QOP_resid_arg_t(1e-20, 0, 0, 0, 0, 0)
        hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
        q.invert(fla, 0.05, hout, hin, ia, ra)
        assert eo_residual(fo, 0.05, q.extract_V(hout, V), src, L, 0) <= 1.05e-20
        its[recon] = ra.final_iter
        q.destroy_V(hin)
        q.destroy_V(hout)
    q.set_opts(prec_sloppy=64, recon_long=1)
    assert its[1] <= 1.1 * its[0] + 10, its
    q.destroy_L(fla)


def _run_multi(q, fla, masses, srcs, rsq, guess=None):
    V = srcs[0].shape[0]
    ras = [[QOP_resid_arg_t(rsq, 0, 0, 0, 0, 0) for _ in ms] for ms in masses]
    hins = [q.create_V(s) for s in srcs]
    houts = [[q.create_V(np.zeros_like(srcs[0]) if guess is None else guess) for _ in ms] for ms in masses]
    ia = QOP_invert_arg_t(1e9, 20000, 20000, 20, 0)
    info = q.invert_multi(fla, masses, houts, hins, ia, ras)
    outs = [[q.extract_V(h, V) for h in row] for row in houts]
    for h in hins:
        q.destroy_V(h)
    for row in houts:
        for h in row:
            q.destroy_V(h)
    return info, ras, outs


@pytest.mark.parametrize("prec", [16, 32])
def test_mixed_multi_mass(prec):
    """Several masses per source (EVEN parity): the sloppy multi-shift CG plus
    per-mass refinement meets every FP64 tolerance, reports the true
    residual, and agrees with the oracle's single-mass solves."""
    L = (8, 8, 8, 8)
    q = gpu_lattice(L, "D")
    fat, lng, _, _ = hisq_links(L, 0.5, 9)
    fo = O.Fla(O.Lattice(L), fat, lng)
    fla = q.create_L_from_raw(fat, lng)
    rsq = 1e-20
    masses = [[0.02, 0.05, 0.1, 0.3, 1.0], [0.2, 0.04]]
    srcs = [LT.gaussian_vector(L, 310 + s) for s in range(2)]
    assert q.set_opts(prec_sloppy=prec) == 0
    info, ras, outs = _run_multi(q, fla, masses, srcs, rsq)
    assert q.set_opts(prec_sloppy=64) == 0
    assert info.status == 0
    for s, ms in enumerate(masses):
        for j, m in enumerate(ms):
            true = eo_residual(fo, m, outs[s][j], srcs[s], L, 0)
            assert true <= rsq * 1.05, (s, m, true)
            assert abs(ras[s][j].final_rsq - true) <= 0.05 * true + 1e-26
            ref, _ = fo.invert(m, srcs[s], O.InvertArg(1e9, 20000, 20000, 5, 0), O.ResidArg(rsq, 0, 0, 0, 0, 0))
            assert rel_norm_err(half(outs[s][j], L, 0), half(ref, L, 0)) <= max(1e-6, 30 * np.sqrt(rsq) / m ** 2)
    q.destroy_L(fla)


@pytest.mark.parametrize("multi_shift", [0, 1])
def test_mixed_multi_mass_iterations(multi_shift):
    """int16 multi-mass solves: batched only (option multi_shift 0: every
    system keeps the iteration count of its own single-mass solve) or
    multi-shift first (the default: fewer iterations than the separate
    solves together, every mass at its FP64 target); a non-zero starting
    guess converges too."""
    L = (8, 8, 8, 8)
    q = gpu_lattice(L, "D")
    fat, lng, _, _ = hisq_links(L, 0.5, 9)
    fo = O.Fla(O.Lattice(L), fat, lng)
    fla = q.create_L_from_raw(fat, lng)
    rsq = 1e-20
    ms = [0.01, 0.03, 0.1, 0.3]
    src = LT.gaussian_vector(L, 320)
    assert q.set_opts(prec_sloppy=16, multi_shift=multi_shift) == 0
    _, ras, _ = _run_multi(q, fla, [ms], [src], rsq)
    its = [r.final_iter for r in ras[0]]
    sep = []
    for m in ms:
        _, r1, _ = _run_multi(q, fla, [[m]], [src], rsq)
        sep.append(r1[0][0].final_iter)
    guess = LT.gaussian_vector(L, 321) * 1e-3
    _, rg, og = _run_multi(q, fla, [ms], [src], rsq, guess=guess)
    assert q.set_opts(prec_sloppy=64, multi_shift=1) == 0   # back to the defaults
    print("multi-mass iterations", its, "separate", sep, "with guess", [r.final_iter for r in rg[0]])
    if multi_shift:
        assert max(its) < 0.9 * sum(sep), (its, sep)
    else:
        for a, b in zip(its, sep):
            assert abs(a - b) <= 0.05 * b + 5, (its, sep)
    for j, m in enumerate(ms):
        assert eo_residual(fo, m, og[0][j], src, L, 0) <= rsq * 1.05
    q.destroy_L(fla)


@pytest.mark.parametrize("bk", [-1, 16])
@pytest.mark.parametrize("L,kind", [((8, 8, 8, 8), "asqtad"), ((4, 4, 4, 8), "hisq")])
def test_mixed_multi_source(L, kind, bk):
    """Many sources, one mass each (some masses repeated, one zero source),
    odd parity: the batched solver (int16 hop, or the tensor-core hop with
    batch_kernel 16) meets every FP64 tolerance, returns m A^{-1} b like the
    oracle, and a zero source gives a zero solution."""
    V = int(np.prod(L))
    q = gpu_lattice(L, "D")
    if kind == "asqtad":
        fat, lng = asqtad_links(L, 0.4, 11)
    else:
        fat, lng, _, _ = hisq_links(L, 0.5, 9)
    fo = O.Fla(O.Lattice(L), fat, lng)
    fla = q.create_L_from_raw(fat, lng)
    rsq = 1e-18
    nsrc = 6
    srcs = [LT.gaussian_vector(L, 400 + s) for s in range(nsrc - 1)]
    srcs.append(np.zeros_like(srcs[0]))
    masses = [[0.03], [0.03], [0.05], [0.08], [0.2], [0.05]]
    assert q.set_opts(prec_sloppy=16, batch_kernel=bk) == 0
    ras = [[QOP_resid_arg_t(rsq, 0, 0, 0, 0, 0)] for _ in range(nsrc)]
    hins = [q.create_V(s) for s in srcs]
    houts = [[q.create_V(np.zeros_like(srcs[0]))] for _ in range(nsrc)]
    ia = QOP_invert_arg_t(1e9, 20000, 20000, 20, 1)
    info = q.invert_multi(fla, masses, houts, hins, ia, ras)
    assert q.set_opts(prec_sloppy=64, batch_kernel=-1) == 0
    assert info.status == 0
    for s in range(nsrc):
        got = q.extract_V(houts[s][0], V)
        m = masses[s][0]
        if s == nsrc - 1:
            assert np.all(half(got, L, 1) == 0) and ras[s][0].final_rsq == 0
            continue
        true = eo_residual(fo, m, got, srcs[s], L, 1)
        assert true <= rsq * 1.05, (s, true)
        assert abs(ras[s][0].final_rsq - true) <= 0.05 * true + 1e-26
        ref, _ = fo.invert(m, srcs[s], O.InvertArg(1e9, 20000, 20000, 5, 1), O.ResidArg(rsq, 0, 0, 0, 0, 0))
        assert rel_norm_err(half(got, L, 1), half(ref, L, 1)) <= max(1e-6, 30 * np.sqrt(rsq) / m ** 2)
    for h in hins:
        q.destroy_V(h)
    for row in houts:
        q.destroy_V(row[0])
    q.destroy_L(fla)


def _single_iters(q, fla, src, m, L, eo=0):
    ia = QOP_invert_arg_t(1e9, 20000, 20000, 5, eo)
    ra = QOP_resid_arg_t(1e-20, 0, 0, 0, 0, 0)
    hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
    info = q.invert(fla, m, hout, hin, ia, ra)
    got = q.extract_V(hout, int(np.prod(L)))
    q.destroy_V(hin)
    q.destroy_V(hout)
    return info.status, ra.final_iter, got


def test_every_hop_kernel_variant():
    """Each selectable int16 hop kernel (option hop_kernel 0-31: plain,
    TMA-staged, register-capped, persistent, cp.async-ring and packed
    FP32x2 forms, the last three with an L2 prefetch of the link stream)
    solves to the FP64 target; the scalar forms share the
    decode and arithmetic order and the packed forms round the scaled site
    components first, so the iteration counts agree within a few per cent."""
    L = (8, 8, 8, 8)
    q = gpu_lattice(L, "D")
    fat, lng, _, _ = hisq_links(L, 0.5, 9)
    fo = O.Fla(O.Lattice(L), fat, lng)
    fla = q.create_L_from_raw(fat, lng)
    src = LT.gaussian_vector(L, 330)
    its = {}
    for v in range(32):
        assert q.set_opts(prec_sloppy=16, hop_kernel=v) == 0
        st, it, got = _single_iters(q, fla, src, 0.03, L)
        assert st == 0
        assert eo_residual(fo, 0.03, got, src, L, 0) <= 1.05e-20, v
        its[v] = it
    assert q.set_opts(hop_kernel=32) != 0                  # out of range
    assert q.set_opts(prec_sloppy=64, hop_kernel=25) == 0
    ref = its[25]
    assert all(abs(i - ref) <= 0.03 * ref + 3 for i in its.values()), its
    q.destroy_L(fla)


def test_fused_update_solves_like_the_four_kernel_iteration():
    """Option fuse_update (packed hop variants 20-26): the second hop also
    reduces <r, Ap> and |Ap|^2 and one kernel updates x, r and p; the
    solves reach the FP64 target with the iteration counts of the
    four-kernel iteration (within rounding noise)."""
    L = (8, 8, 8, 8)
    q = gpu_lattice(L, "D")
    fat, lng, _, _ = hisq_links(L, 0.5, 9)
    fo = O.Fla(O.Lattice(L), fat, lng)
    fla = q.create_L_from_raw(fat, lng)
    try:
        for v in (20, 23, 25):
            its = []
            for fuse in (0, 1):
                assert q.set_opts(prec_sloppy=16, hop_kernel=v, fuse_update=fuse) == 0
                for eo, mass, seed in ((0, 0.03, 331), (1, 0.01, 332)):
                    src = LT.gaussian_vector(L, seed)
                    st, it, got = _single_iters(q, fla, src, mass, L, eo)
                    assert st == 0
                    assert eo_residual(fo, mass, got, src, L, eo) <= 1.05e-20, (v, fuse, eo)
                    its.append(it)
            assert all(abs(a - b) <= 0.03 * b + 3 for a, b in zip(its[2:], its[:2])), (v, its)
    finally:
        assert q.set_opts(prec_sloppy=64, hop_kernel=25, fuse_update=1) == 0
        q.destroy_L(fla)


def test_programmatic_dependent_launch_solves_like_the_default():
    """Option pdl: the three kernels of the fused int16 iteration launched
    as programmatic dependents (each waits in griddepcontrol.wait for the one
    ahead of it) compute exactly what the ordinary launches compute: the
    same iteration count and the same solution, bit for bit."""
    L = (8, 8, 8, 8)
    q = gpu_lattice(L, "D")
    fat, lng, _, _ = hisq_links(L, 0.5, 9)
    fo = O.Fla(O.Lattice(L), fat, lng)
    fla = q.create_L_from_raw(fat, lng)
    src = LT.gaussian_vector(L, 331)
    try:
        out = {}
        for pdl in (0, 1, 0, 1):
            assert q.set_opts(prec_sloppy=16, hop_kernel=25, fuse_update=1, pdl=pdl) == 0
            st, it, got = _single_iters(q, fla, src, 0.03, L)
            assert st == 0 and eo_residual(fo, 0.03, got, src, L, 0) <= 1.05e-20
            if pdl in out:
                assert it == out[pdl][0] and np.array_equal(got, out[pdl][1])
            out[pdl] = (it, got)
        assert out[1][0] == out[0][0] and np.array_equal(out[1][1], out[0][1])
    finally:
        assert q.set_opts(prec_sloppy=64, pdl=1) == 0
        q.destroy_L(fla)


def test_every_batch_kernel_variant():
    """Each selectable batched hop (option batch_kernel 0-15 on int16 vectors,
    16 the tensor-core hop on bf16 hi / lo vectors) solves a four-source
    batch to the FP64 target with the iteration counts of the default
    variant."""
    L = (8, 8, 8, 8)
    q = gpu_lattice(L, "D")
    fat, lng = asqtad_links(L, 0.4, 11)
    fo = O.Fla(O.Lattice(L), fat, lng)
    fla = q.create_L_from_raw(fat, lng)
    srcs = [LT.gaussian_vector(L, 340 + s) for s in range(4)]
    ms = [[0.03], [0.05], [0.03], [0.1]]
    its = {}
    for v in range(17):
        assert q.set_opts(prec_sloppy=16, batch_kernel=v) == 0
        info, ras, outs = _run_multi(q, fla, ms, srcs, 1e-20)
        assert info.status == 0
        for s in range(4):
            assert eo_residual(fo, ms[s][0], outs[s][0], srcs[s], L, 0) <= 1.05e-20, (v, s)
        its[v] = [r[0].final_iter for r in ras]
    assert q.set_opts(batch_kernel=17) != 0
    assert q.set_opts(prec_sloppy=64, batch_kernel=-1) == 0
    print("batched iterations per variant", its)
    for v, it in its.items():
        assert all(abs(a - b) <= 0.03 * b + 3 for a, b in zip(it, its[7])), its
    q.destroy_L(fla)


def test_autotuned_hop_variants():
    """Options hop_kernel -1 and batch_kernel -2: the first solve on a
    lattice times the candidate variants (one-system hops 20-26; batched
    hops 1, 6, 7, 9, 12) and keeps the fastest; the solves reach the FP64
    target with the iteration counts of the fixed defaults, and a second
    solve (cached choice) repeats the first."""
    L = (8, 8, 8, 8)
    q = gpu_lattice(L, "D")
    fat, lng, _, _ = hisq_links(L, 0.5, 9)
    fo = O.Fla(O.Lattice(L), fat, lng)
    fla = q.create_L_from_raw(fat, lng)
    src = LT.gaussian_vector(L, 330)
    srcs = [LT.gaussian_vector(L, 340 + s) for s in range(4)]
    ms = [[0.03], [0.05], [0.03], [0.1]]
    assert q.set_opts(hop_kernel=-2) != 0 and q.set_opts(batch_kernel=-3) != 0
    try:
        assert q.set_opts(prec_sloppy=16, hop_kernel=25, batch_kernel=-1) == 0
        ref_it = _single_iters(q, fla, src, 0.03, L)[1]
        info, ras, _ = _run_multi(q, fla, ms, srcs, 1e-20)
        ref_b = [r[0].final_iter for r in ras]
        assert q.set_opts(hop_kernel=-1, batch_kernel=-2) == 0
        runs = []
        for _ in range(2):
            st, it, got = _single_iters(q, fla, src, 0.03, L)
            assert st == 0 and eo_residual(fo, 0.03, got, src, L, 0) <= 1.05e-20
            info, ras, outs = _run_multi(q, fla, ms, srcs, 1e-20)
            assert info.status == 0
            for s in range(4):
                assert eo_residual(fo, ms[s][0], outs[s][0], srcs[s], L, 0) <= 1.05e-20, s
            runs.append((it, [r[0].final_iter for r in ras]))
        assert runs[0] == runs[1]
        assert abs(runs[0][0] - ref_it) <= 0.03 * ref_it + 3, (runs, ref_it)
        assert all(abs(a - b) <= 0.03 * b + 3 for a, b in zip(runs[0][1], ref_b)), (runs, ref_b)
    finally:
        assert q.set_opts(prec_sloppy=64, hop_kernel=25, batch_kernel=-1) == 0
        q.destroy_L(fla)


@pytest.mark.parametrize("L", [(6, 6, 6, 6), (4, 6, 4, 10)])
def test_mixed_ragged_site_blocks(L):
    """Lattices whose sites per parity are not a multiple of the 128-site
    link blocks (padded last block): single-system and batched int16 solves
    both meet the FP64 target and agree with the oracle."""
    V = int(np.prod(L))
    q = gpu_lattice(L, "D")
    fat, lng, _, _ = hisq_links(L, 0.5, 9)
    fo = O.Fla(O.Lattice(L), fat, lng)
    fla = q.create_L_from_raw(fat, lng)
    srcs = [LT.gaussian_vector(L, 700 + s) for s in range(3)]
    assert q.set_opts(prec_sloppy=16) == 0
    st, _, got = _single_iters(q, fla, srcs[0], 0.05, L)
    assert st == 0 and eo_residual(fo, 0.05, got, srcs[0], L, 0) <= 1.05e-20
    for bk in (-1, 16):      # int16 and tensor-core batched hops
        assert q.set_opts(batch_kernel=bk) == 0
        info, ras, outs = _run_multi(q, fla, [[0.05], [0.1], [0.05]], srcs, 1e-20)
        assert info.status == 0
        for s, m in enumerate([0.05, 0.1, 0.05]):
            assert eo_residual(fo, m, outs[s][0], srcs[s], L, 0) <= 1.05e-20
            ref, _ = fo.invert(m, srcs[s], O.InvertArg(1e9, 20000, 20000, 5, 0), O.ResidArg(1e-20, 0, 0, 0, 0, 0))
            assert rel_norm_err(half(outs[s][0], L, 0), half(ref, L, 0)) <= max(1e-6, 30 * 1e-10 / m ** 2)
    assert q.set_opts(prec_sloppy=64, batch_kernel=-1) == 0
    q.destroy_L(fla)


@pytest.mark.parametrize("multi_shift", [0, 1])
def test_batch_tail_handoff_meets_targets(multi_shift):
    """Option batch_tail: the last system running in a batch finishes in the
    one-system solver (the correction A e = b - A x from its current x).
    With and without the hand-off every mass meets its FP64 target (checked
    with the oracle), and the hand-off costs the handed-off system no more
    than a few percent of iterations."""
    L = (8, 8, 8, 8)
    q = gpu_lattice(L, "D")
    fat, lng, _, _ = hisq_links(L, 0.5, 9)
    fo = O.Fla(O.Lattice(L), fat, lng)
    fla = q.create_L_from_raw(fat, lng)
    rsq = 1e-20
    ms = [0.01, 0.05, 0.2]
    src = LT.gaussian_vector(L, 330)
    its = {}
    try:
        for tail in (0, 1):
            assert q.set_opts(prec_sloppy=16, multi_shift=multi_shift, batch_tail=tail) == 0
            _, ras, outs = _run_multi(q, fla, [ms], [src], rsq)
            its[tail] = [r.final_iter for r in ras[0]]
            for j, m in enumerate(ms):
                true = eo_residual(fo, m, outs[0][j], src, L, 0)
                assert true <= rsq * 1.05, (tail, m, true)
                assert abs(ras[0][j].final_rsq - true) <= 0.05 * true + 1e-26
    finally:
        assert q.set_opts(prec_sloppy=64, multi_shift=1, batch_tail=1) == 0
    print("iterations without / with the hand-off", its)
    assert max(its[1]) <= 1.1 * max(its[0]) + 20, its
    q.destroy_L(fla)
