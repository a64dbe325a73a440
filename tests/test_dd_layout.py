"""Decomposition host logic on CPU (no GPU): the reference's split of the
lattice over processes (lib/layout_user.c:110-165), node numbers and
node-local raw indices (:225-258), neighbour ranks, and the halo layout of
the decomposed hop.  A world-size-2 gloo job packs halos in the documented
layout (slab, colour, face site = floor(lex'/2)), pairs the sends and
receives in the library's posting order with the library's neighbour ranks,
and checks every received element against the global field at the halo
coordinates."""
import itertools
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from qopqdp_b200 import qop  # noqa: E402


@pytest.mark.parametrize("L,n,want", [
    # traced by hand through layout_user.c:110-165
    ((32, 32, 32, 64), 8, (1, 1, 2, 4)),
    ((8, 8, 8, 8), 16, (2, 2, 2, 2)),
    ((24, 24, 24, 48), 12, (1, 2, 2, 3)),
    ((16, 16, 16, 16), 6, (1, 1, 2, 3)),   # 3 divides no extent: the longest direction takes it
    ((8, 8, 8, 8), 1, (1, 1, 1, 1)),
])
def test_layout_hyper_matches_reference_split(L, n, want):
    assert qop.layout_hyper(L, n) == want


@pytest.mark.parametrize("L,P", [((4, 4, 8, 8), (1, 1, 2, 2)), ((8, 4, 4, 12), (2, 1, 1, 3)), ((4, 4, 4, 4), (1, 1, 1, 1))])
def test_node_number_and_index_partition_the_lattice(L, P):
    nr = int(np.prod(P))
    b = [L[i] // P[i] for i in range(4)]
    vloc = int(np.prod(b))
    seen = {r: set() for r in range(nr)}
    for x in itertools.product(*[range(n) for n in L]):
        r = qop.layout_node_number(L, P, x)
        i = qop.layout_node_index(L, P, x)
        assert 0 <= r < nr and 0 <= i < vloc
        # rank from block coordinates, direction 0 fastest
        m = [x[k] // b[k] for k in range(4)]
        assert r == m[0] + P[0] * (m[1] + P[1] * (m[2] + P[2] * m[3]))
        # node-local raw order: the block's own even-first lexicographic order
        loc = [x[k] - m[k] * b[k] for k in range(4)]
        lex = ((loc[0] * b[1] + loc[1]) * b[2] + loc[2]) * b[3] + loc[3]
        assert i == (lex // 2 if sum(x) % 2 == 0 else (lex + vloc) // 2)
        assert i not in seen[r]
        seen[r].add(i)
    assert all(len(s) == vloc for s in seen.values())


def test_neighbors_are_symmetric():
    P = (2, 1, 3, 4)
    nr = int(np.prod(P))
    for r in range(nr):
        nb = qop.layout_neighbors(P, r)
        for mu, (dn, up) in enumerate(nb):
            assert qop.layout_neighbors(P, up)[mu][0] == r
            assert qop.layout_neighbors(P, dn)[mu][1] == r
            if P[mu] == 1:
                assert dn == up == r


# ---------------------------------------------------------------- halo exchange
GL = (4, 4, 8, 4)
NL = 16


def global_fields():
    rng = np.random.default_rng(17)
    psi = rng.standard_normal(GL + (3, 2)) @ np.array([1, 1j])
    fat = rng.standard_normal((4,) + GL + (3, 3, 2)) @ np.array([1, 1j])
    lng = rng.standard_normal((4,) + GL + (3, 3, 2)) @ np.array([1, 1j])
    return psi, fat, lng


def face_site(b, mu, xm, q, fi):
    """Local coordinates of face site fi of parity q on the slab x_mu = xm."""
    others = [nu for nu in range(4) if nu != mu]
    x = [0] * 4
    rem = 2 * fi
    for nu in reversed(others):
        x[nu] = rem % b[nu]
        rem //= b[nu]
    x[mu] = xm
    if sum(x) % 2 != q:
        x[others[-1]] += 1
    return x


def _exchange_worker(rank, world, port, q_out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        P = qop.layout_hyper(GL, world)
        b = [GL[i] // P[i] for i in range(4)]
        m = [0] * 4
        r = rank
        for i in range(4):
            m[i] = r % P[i]
            r //= P[i]
        O = [m[i] * b[i] for i in range(4)]
        nb = qop.layout_neighbors(P, rank)
        psi, fat, lng = global_fields()

        def gpos(x):
            return tuple((O[i] + x[i]) % GL[i] for i in range(4))

        errors = 0
        for parity in (0, 1):
            for mu in range(4):
                if P[mu] == 1:
                    continue
                fh = int(np.prod(b)) // b[mu] // 2
                # pack: raw slabs x_mu = s; products -U^+ psi at x_mu = L-1 (fat), L-1-j (long)
                raw = np.zeros((3, 3, fh), complex)
                prod = np.zeros((4, 3, fh), complex)
                for fi in range(fh):
                    for s in range(3):
                        raw[s, :, fi] = psi[gpos(face_site(b, mu, s, parity, fi))]
                    for j in range(4):
                        xm = b[mu] - 1 - (0 if j == 0 else j - 1)
                        y = gpos(face_site(b, mu, xm, parity, fi))
                        U = (fat if j == 0 else lng)[(mu,) + y]
                        prod[j, :, fi] = -U.conj().T @ psi[y]
                up = np.zeros_like(raw)
                dn = np.zeros_like(prod)
                # the library's posting order: raw to -mu, up from +mu, products to +mu, down from -mu
                reqs = []
                for buf, peer, send in ((raw, nb[mu][0], True), (up, nb[mu][1], False),
                                        (prod, nb[mu][1], True), (dn, nb[mu][0], False)):
                    t = torch.from_numpy(buf.view(np.float64))
                    reqs.append((dist.isend if send else dist.irecv)(t, peer, tag=0))
                for rq in reqs:
                    rq.wait()
                # check against the global field at the halo coordinates of the
                # output sites (parity 1 - parity) next to each face
                for fi in range(fh):
                    for j in range(3):
                        # up halo slab j: the site x_mu = L + j with the face coordinates of index fi
                        x = face_site(b, mu, b[mu] + j, parity, fi)
                        errors += not np.allclose(up[j, :, fi], psi[gpos(x)], rtol=0, atol=0)
                    for s in range(4):
                        xm = -1 if s == 0 else -s
                        y = gpos(face_site(b, mu, xm, parity, fi))
                        U = (fat if s == 0 else lng)[(mu,) + y]
                        errors += not np.allclose(dn[s, :, fi], -U.conj().T @ psi[y], rtol=0, atol=0)
        dist.barrier()
        q_out.put((rank, P, errors))
    finally:
        dist.destroy_process_group()


def test_two_process_halo_exchange_layout():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + os.getpid() % 1000
    ps = [ctx.Process(target=_exchange_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=180) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, P, errors in res:
        assert P == (1, 1, 2, 1)
        assert errors == 0, (rank, errors)


# ---------------------------------------------------------------- the library's halo plan
def _plan_hop_worker(rank, world, port, GLb, P, q_out):
    """One rank of the decomposed hop, assembled on the CPU from the
    library's own plan: node numbers and node-local raw indices
    (QOPB_layout_node_number / _node_index), neighbour ranks
    (QOPB_layout_neighbors), the packed halo sites and link slots
    (QOPB_dd_pack_site) and where each boundary term reads its halo
    (QOPB_dd_halo_ref).  The result on the rank's sites is compared with the
    oracle's Dslash of the global field."""
    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from qopqdp_b200 import lattice as LT
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        GL = tuple(GLb)
        b = tuple(GL[i] // P[i] for i in range(4))
        Vg, Vl = int(np.prod(GL)), int(np.prod(b))
        rng = np.random.default_rng(23)
        psi = rng.standard_normal((Vg, 3, 2))
        fat = [rng.standard_normal((Vg, 3, 3, 2)) for _ in range(4)]
        lng = [rng.standard_normal((Vg, 3, 3, 2)) for _ in range(4)]
        cz = lambda a: a[..., 0] + 1j * a[..., 1]
        psic, fatc, lngc = cz(psi), [cz(a) for a in fat], [cz(a) for a in lng]
        xs = LT.raw_coords(GL)
        # this rank's sites, in its node-local raw order
        loc = {}
        for g in range(Vg):
            x = tuple(int(v) for v in xs[g])
            if qop.layout_node_number(GL, P, x) == rank:
                loc[qop.layout_node_index(GL, P, x)] = g
        assert sorted(loc) == list(range(Vl))
        lg = np.array([loc[i] for i in range(Vl)])           # local raw index -> global raw index
        origin = xs[lg].min(axis=0)
        assert all(o % 2 == 0 for o in origin)
        lraw = {tuple(int(v) for v in xs[g] - origin): i for i, g in enumerate(lg)}
        nb = qop.layout_neighbors(P, rank)
        ref_fla = O.Fla(O.Lattice(GL), fat, lng)
        errs = []
        for p in (0, 1):
            q = 1 - p
            up, dn = {}, {}
            for mu in range(4):
                if P[mu] == 1:
                    continue
                fh = Vl // b[mu] // 2
                sraw = np.zeros((3, 3, fh), complex)
                sprod = np.zeros((4, 3, fh), complex)
                for s in range(7):
                    for fi in range(fh):
                        x, slot = qop.dd_pack_site(b, mu, 16, q, s, fi)
                        assert sum(x) % 2 == q
                        g = lg[lraw[x]]
                        if slot < 0:
                            sraw[s, :, fi] = psic[g]
                        else:
                            U = (fatc if slot == 4 * mu else lngc)[mu][g] * 0.5
                            sprod[s - 3, :, fi] = -U.conj().T @ psic[g]
                gup, gdn = np.zeros_like(sraw), np.zeros_like(sprod)
                reqs = []
                for buf, peer, send, tag in ((sraw, nb[mu][0], True, 1), (gup, nb[mu][1], False, 1),
                                             (sprod, nb[mu][1], True, 2), (gdn, nb[mu][0], False, 2)):
                    t = torch.from_numpy(buf.view(np.float64))
                    reqs.append((dist.isend if send else dist.irecv)(t, peer, tag=tag))
                for rq in reqs:
                    rq.wait()
                up[mu], dn[mu] = gup, gdn
            want = cz(ref_fla.dslash(0.0, psi, p, q))
            worst = 0.0
            for i in range(Vl):
                x = tuple(int(v) for v in xs[lg[i]] - origin)
                if sum(x) % 2 != p:
                    continue
                acc = np.zeros(3, complex)
                for mu in range(4):
                    for d in (1, 3, -1, -3):
                        # directions that are not split wrap inside the block
                        where = qop.dd_halo_ref(b, x, mu, d) if P[mu] > 1 else None
                        U_here = (fatc if abs(d) == 1 else lngc)[mu][lg[i]] * 0.5
                        if where is None:
                            y = list(x)
                            y[mu] = (y[mu] + d) % b[mu]
                            gy = lg[lraw[tuple(y)]]
                            if d > 0:
                                acc += U_here @ psic[gy]
                            else:
                                U = (fatc if d == -1 else lngc)[mu][gy] * 0.5
                                acc -= U.conj().T @ psic[gy]
                        elif where[0] == "up":
                            acc += U_here @ up[mu][where[1], :, where[2]]
                        else:
                            acc += dn[mu][where[1], :, where[2]]
                w = want[lg[i]]
                worst = max(worst, float(np.abs(acc - w).max() / np.abs(w).max()))
            errs.append(worst)
        dist.barrier()
        q_out.put((rank, errs))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("GL,P", [((4, 4, 4, 8), (1, 1, 1, 2)), ((8, 4, 4, 4), (2, 1, 1, 1)),
                                  ((4, 8, 6, 4), (1, 2, 1, 1))])
def test_two_process_hop_through_library_halo_plan(GL, P):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + (os.getpid() + 7 * P.index(2)) % 1000
    ps = [ctx.Process(target=_plan_hop_worker, args=(r, 2, port, GL, P, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = []
    import queue
    import time
    t0 = time.time()
    while len(res) < len(ps):
        try:
            res.append(q.get(timeout=2))
        except queue.Empty:
            # a rank that died (an exception) ends the test instead of a wait
            assert all(p.exitcode in (None, 0) for p in ps), [p.exitcode for p in ps]
            assert time.time() - t0 < 300
    res.sort()
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, errs in res:
        assert max(errs) < 1e-14, (rank, errs)


def test_halo_plan_hooks_reject_bad_arguments():
    with pytest.raises(ValueError):
        qop.dd_pack_site((4, 4, 4, 5), 0, 16, 0, 0, 0)       # odd extent
    with pytest.raises(ValueError):
        qop.dd_pack_site((4, 4, 4, 4), 0, 16, 0, 7, 0)       # slab past depth + products
    with pytest.raises(ValueError):
        qop.dd_pack_site((4, 4, 4, 4), 0, 16, 0, 0, 32)      # face past fh
    with pytest.raises(ValueError):
        qop.dd_halo_ref((4, 4, 4, 4), (0, 0, 0, 4), 3, 1)    # site outside the block
    with pytest.raises(ValueError):
        qop.dd_halo_ref((4, 4, 4, 4), (0, 0, 0, 0), 3, 2)    # not a hop displacement
    assert qop.dd_halo_ref((4, 4, 4, 4), (1, 1, 1, 1), 3, 1) is None
    assert qop.dd_halo_ref((4, 4, 4, 4), (1, 1, 1, 3), 3, 3)[0:2] == ("up", 2)
    assert qop.dd_halo_ref((4, 4, 4, 4), (1, 1, 1, 0), 3, -3)[0:2] == ("dn", 3)
