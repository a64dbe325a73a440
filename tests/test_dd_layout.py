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
