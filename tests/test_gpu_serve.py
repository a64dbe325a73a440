"""Several lattices in one process and the solve service (QOPB_lattice_*,
QOPB_serve_*): handles are tied to the lattice they were created on, and
queued requests on two resident lattices are solved in batches to their
FP64 targets with the QOP_asqtad_invert normalisation."""
import numpy as np
import pytest

import oracle as O
from conftest import gpu_lattice
from helpers import hisq_links, asqtad_links, eo_residual, rel_norm_err, half, site_rel_err
from qopqdp_b200 import lattice as LT
from qopqdp_b200.qop import QOP_info_t

pytestmark = pytest.mark.gpu

LA = (4, 4, 4, 8)
LB = (8, 8, 8, 8)


def test_handles_belong_to_their_lattice():
    q = gpu_lattice(LA, "D")
    lb = q.lattice_create(LB)
    assert lb >= 1
    assert q.lattice_create((4, 4, 4, 5)) == -1          # odd extent refused
    assert q.lattice_use(99) == -1
    VB = int(np.prod(LB))
    fat, lng = asqtad_links(LB, 0.3, 7)
    fo = O.Fla(O.Lattice(LB), fat, lng)
    assert q.lattice_use(lb) == 0
    fla = q.create_L_from_raw(fat, lng)
    src = LT.gaussian_vector(LB, 500)
    hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
    # on lattice 0 the lattice-B handles are refused, nothing runs
    assert q.lattice_use(0) == 0
    info = q.dslash(fla, 0.1, hout, hin, 2, 2)
    assert info.status != 0
    # on their own lattice they work and match the oracle
    assert q.lattice_use(lb) == 0
    info = q.dslash(fla, 0.1, hout, hin, 2, 2)
    assert info.status == 0
    ref = fo.dslash(0.1, src, 2, 2)
    assert site_rel_err(q.extract_V(hout, VB), ref) <= 1e-13
    q.destroy_V(hin)
    q.destroy_V(hout)
    q.destroy_L(fla)
    assert q.lattice_use(0) == 0


@pytest.mark.parametrize("policy", [0, 1])
def test_serve_two_lattices(policy):
    """Queued requests on two lattices, both service policies (0: every
    engine steps in turn; 1: the engine holding the oldest request)."""
    q = gpu_lattice(LA, "D")
    assert q.set_opts(serve_policy=2) != 0
    assert q.set_opts(serve_policy=policy) == 0
    lb = q.lattice_create(LB)
    fa, la_, _, _ = hisq_links(LA, 0.5, 9)
    fb, lb_ = asqtad_links(LB, 0.3, 7)
    foa, fob = O.Fla(O.Lattice(LA), fa, la_), O.Fla(O.Lattice(LB), fb, lb_)
    assert q.lattice_use(0) == 0
    ha = q.create_L_from_raw(fa, la_)
    assert q.lattice_use(lb) == 0
    hb = q.create_L_from_raw(fb, lb_)
    assert q.lattice_use(0) == 0
    rng = np.random.default_rng(11)
    reqs = []
    for r in range(10):
        on_b = r % 2 == 1
        L = LB if on_b else LA
        nrhs = int(rng.integers(1, 4))
        srcs = [LT.gaussian_vector(L, 600 + 10 * r + k) for k in range(nrhs)]
        dsts = [np.zeros_like(s) for s in srcs]
        mass = float(np.exp(rng.uniform(np.log(0.02), np.log(0.2))))
        rsq = 1e-20 if r % 3 else 1e-16
        eo = r % 2 if r < 6 else 1 - r % 2
        reqs.append((on_b, L, srcs, dsts, mass, rsq, eo))
    assert q.serve_start() == 0
    assert q.serve_start() == -1                      # already running
    bad = q.serve_submit(ha, 0, 0, 0.1, 1e-20, [], [])
    assert bad == -1                                  # no sources
    tickets = [q.serve_submit(hb if on_b else ha, lb if on_b else 0, eo, mass, rsq, srcs, dsts)
               for (on_b, L, srcs, dsts, mass, rsq, eo) in reqs]
    assert all(t >= 0 for t in tickets)
    results = []
    for t in tickets:
        rc, res = q.serve_wait(t, 120.0)
        assert rc == 0
        results.append(res)
    assert q.serve_wait(tickets[0], 1.0)[0] == -1      # released
    assert q.serve_stop() == 0
    assert q.set_opts(serve_policy=0) == 0
    for (on_b, L, srcs, dsts, mass, rsq, eo), res in zip(reqs, results):
        fo = fob if on_b else foa
        assert res.status == 0
        assert res.batch_systems >= len(srcs)
        assert res.total_ms >= res.solve_ms >= 0
        assert res.final_rsq_max <= rsq * 1.05
        for s, d in zip(srcs, dsts):
            true = eo_residual(fo, mass, d, s, L, eo)
            assert true <= rsq * 1.05, (L, mass, rsq, true)
    # one solution against the oracle's solve of the same system
    on_b, L, srcs, dsts, mass, rsq, eo = reqs[1]
    ref, _ = fob.invert(mass, srcs[0], O.InvertArg(1e9, 20000, 20000, 5, eo), O.ResidArg(rsq, 0, 0, 0, 0, 0))
    assert rel_norm_err(half(dsts[0], L, eo), half(ref, L, eo)) <= max(1e-6, 30 * np.sqrt(rsq) / mass ** 2)
    assert q.lattice_use(lb) == 0
    q.destroy_L(hb)
    assert q.lattice_use(0) == 0
    q.destroy_L(ha)


def test_serve_continuous_batching_same_alone_and_in_the_mix():
    """Continuous batching: a request that arrives while a long request on
    the same links is in flight joins its batch at once (it shares A's hop
    launches and finishes long before A), a request on another lattice runs
    beside them, and each result is the same alone and in the mix (both meet
    the FP64 target; their difference is within the solve tolerance)."""
    import time
    q = gpu_lattice(LA, "D")
    lb = q.lattice_create(LB)
    fa, la_, _, _ = hisq_links(LA, 0.5, 9)
    fb, lb_ = asqtad_links(LB, 0.3, 7)
    foa, fob = O.Fla(O.Lattice(LA), fa, la_), O.Fla(O.Lattice(LB), fb, lb_)
    assert q.lattice_use(0) == 0
    ha = q.create_L_from_raw(fa, la_)
    assert q.lattice_use(lb) == 0
    hb = q.create_L_from_raw(fb, lb_)
    assert q.lattice_use(0) == 0
    rsq = 1e-20
    # A: 4 sources at m = 0.002 on LB (~16k iterations); R: LB, same links
    # and parity, m = 0.05; C: LA, m = 0.1
    a_src = [LT.gaussian_vector(LB, 700 + k) for k in range(4)]
    r_src, c_src = LT.gaussian_vector(LB, 710), LT.gaussian_vector(LA, 711)
    R = (hb, lb, 0, 0.05)
    Cq = (ha, 0, 1, 0.1)
    assert q.serve_start() == 0
    try:
        alone = {}
        for name, (h, lat, eo, m), s in (("R", R, r_src), ("C", Cq, c_src)):
            d = [np.zeros_like(s)]
            rc, res = q.serve_wait(q.serve_submit(h, lat, eo, m, rsq, [s], d), 120.0)
            assert rc == 0 and res.status == 0 and res.batch_systems == 1
            alone[name] = (d[0], res.iters_max)
        a_dst = [np.zeros_like(s) for s in a_src]
        r_dst, c_dst = [np.zeros_like(r_src)], [np.zeros_like(c_src)]
        t_a = time.perf_counter()
        ta = q.serve_submit(hb, lb, 0, 0.002, rsq, a_src, a_dst)
        assert ta >= 0
        assert q.serve_wait(ta, 0.05)[0] == 1          # A is in flight
        t_r = time.perf_counter()
        tr = q.serve_submit(*R[:3], R[3], rsq, [r_src], r_dst)
        tc = q.serve_submit(*Cq[:3], Cq[3], rsq, [c_src], c_dst)
        rc_r, res_r = q.serve_wait(tr, 120.0)
        rc_c, res_c = q.serve_wait(tc, 120.0)
        rc_a, res_a = q.serve_wait(ta, 300.0)
    finally:
        assert q.serve_stop() == 0
    assert rc_r == rc_c == rc_a == 0
    assert res_r.status == res_c.status == res_a.status == 0
    # R shared A's batch and did not wait for it
    assert res_r.batch_systems >= 5, res_r.batch_systems
    assert res_r.queue_ms < 0.25 * res_a.solve_ms, (res_r.queue_ms, res_a.solve_ms)
    assert 1e3 * (t_r - t_a) + res_r.total_ms < res_a.total_ms, (res_r.total_ms, res_a.total_ms)
    assert 1e3 * (t_r - t_a) + res_c.total_ms < res_a.total_ms, (res_c.total_ms, res_a.total_ms)
    # every result meets its FP64 target
    for fo, L, eo, m, srcs, dsts in ((fob, LB, 0, 0.002, a_src, a_dst), (fob, LB, 0, 0.05, [r_src], r_dst),
                                     (foa, LA, 1, 0.1, [c_src], c_dst)):
        for s, d in zip(srcs, dsts):
            assert eo_residual(fo, m, d, s, L, eo) <= rsq * 1.05, (L, m)
    # the same alone and in the mix
    for name, L, eo, m, d in (("R", LB, 0, 0.05, r_dst[0]), ("C", LA, 1, 0.1, c_dst[0])):
        d0, it0 = alone[name]
        err = rel_norm_err(half(d, L, eo), half(d0, L, eo))
        assert err <= max(1e-8, 30 * np.sqrt(rsq) / m ** 2), (name, err)
    assert abs(res_r.iters_max - alone["R"][1]) <= 2
    assert abs(res_c.iters_max - alone["C"][1]) <= 2
    assert q.lattice_use(lb) == 0
    q.destroy_L(hb)
    assert q.lattice_use(0) == 0
    q.destroy_L(ha)
