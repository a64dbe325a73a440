"""QOPB_D3_asqtad_ddagd_norm2_noalloc through the C ABI.

This entry point serves callers that cannot allocate device memory where
they apply the operator: applications whose own caching allocator has
reserved the GPU's memory up front (a cudaMalloc from this library fails
there), and loops that must not wait on an allocator.  Its result must
equal the allocating QOP_D3_asqtad_ddagd_norm2 on two calls in a row (the
scratch it reuses keeps the previous call's contents), it must allocate
nothing, it must refuse handles that are dead or belong to another lattice,
and lattices beyond its fixed scratch must be rejected.  Collected last so
a failure here cannot hide other tests; it also passes when run alone in a
fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import gpu_lattice
from devmem import Memory
from helpers import asqtad_links, site_rel_err
from qopqdp_b200 import lattice as LT
from qopqdp_b200.qop import QOP_info_t

pytestmark = pytest.mark.gpu

NOALLOC_MAX_VH = 65536


def _fn(q):
    f = q.lib.QOPB_D3_asqtad_ddagd_norm2_noalloc
    f.argtypes = [C.POINTER(QOP_info_t), C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_int]
    f.restype = C.c_double
    return f


def _launches(q):
    q.lib.QOPB_launch_count.restype = C.c_ulonglong
    return int(q.lib.QOPB_launch_count())


def _check_against_allocating(q, L, mass, seed, calls=2):
    V = int(np.prod(L))
    fn = _fn(q)
    fat, lng = asqtad_links(L, 0.3, seed)
    fla = q.create_L_from_raw(fat, lng)
    for eo in (0, 1):
        src = LT.gaussian_vector(L, 200 + eo)
        hin = q.create_V(src)
        href = q.create_V(np.zeros_like(src))
        n_ref = q.ddagd_norm2(fla, mass, href, hin, eo)
        ref = q.extract_V(href, V)
        for call in range(calls):                   # scratch reused between calls
            hout = q.create_V(np.zeros_like(src))
            info = QOP_info_t()
            n = fn(C.byref(info), fla, mass, hout, hin, eo)
            got = q.extract_V(hout, V)
            assert info.status == 0
            assert abs(n - n_ref) <= 1e-13 * abs(n_ref), (call, n, n_ref)
            assert site_rel_err(got, ref) <= 1e-13, call
            q.destroy_V(hout)
        q.destroy_V(hin)
        q.destroy_V(href)
    q.destroy_L(fla)


def test_noalloc_ddagd_norm2_matches_allocating_entry_point():
    L = (8, 8, 8, 8)
    q = gpu_lattice(L, "D")
    _check_against_allocating(q, L, 0.05, 7)


def test_noalloc_at_its_maximum_lattice():
    L = (16, 16, 16, 32)                             # exactly 65536 sites per parity
    assert int(np.prod(L)) // 2 == NOALLOC_MAX_VH
    q = gpu_lattice(L, "D")
    _check_against_allocating(q, L, 0.1, 11)


def test_noalloc_allocates_nothing():
    L = (8, 8, 8, 8)
    V = int(np.prod(L))
    q = gpu_lattice(L, "D")
    fn = _fn(q)
    fat, lng = asqtad_links(L, 0.3, 7)
    fla = q.create_L_from_raw(fat, lng)
    src = LT.gaussian_vector(L, 300)
    hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
    info = QOP_info_t()
    assert fn(C.byref(info), fla, 0.05, hout, hin, 0) > 0      # first call: scratch address lookup
    mem = Memory()
    # the measurement sees the allocating entry point's temporary
    used0 = mem.used()
    mem.reset_high()
    q.ddagd_norm2(fla, 0.05, hout, hin, 0)
    assert mem.high() >= used0 + 3 * 16 * (V // 2), "pool high-water mark missed a temporary vector"
    # and the no-alloc entry point leaves both the pool and free memory alone
    used1, free1 = mem.used(), mem.free()
    mem.reset_high()
    for _ in range(4):
        assert fn(C.byref(info), fla, 0.05, hout, hin, 0) > 0 and info.status == 0
    assert mem.high() == used1 and mem.used() == used1
    assert mem.free() == free1
    for h in (hin, hout):
        q.destroy_V(h)
    q.destroy_L(fla)


def test_noalloc_refuses_foreign_and_dead_handles():
    L = (8, 8, 8, 8)
    LB = (4, 4, 4, 8)
    q = gpu_lattice(L, "D")
    fn = _fn(q)
    fat, lng = asqtad_links(L, 0.3, 7)
    fla = q.create_L_from_raw(fat, lng)
    src = LT.gaussian_vector(L, 400)
    hin, hout = q.create_V(src), q.create_V(np.zeros_like(src))
    # handles made on a second, smaller lattice
    lb = q.lattice_create(LB)
    assert lb >= 1 and q.lattice_use(lb) == 0
    fb, lb_ = asqtad_links(LB, 0.3, 7)
    fla_b = q.create_L_from_raw(fb, lb_)
    vb = q.create_V(LT.gaussian_vector(LB, 401))
    assert q.lattice_use(0) == 0
    dead = q.create_V(src)
    q.destroy_V(dead)
    cases = [(fla_b, hout, hin), (fla, vb, hin), (fla, hout, vb), (fla, hout, dead), (fla, dead, hin), (None, hout, hin)]
    for args in cases:
        n0 = _launches(q)
        info = QOP_info_t()
        n = fn(C.byref(info), args[0], 0.05, args[1], args[2], 0)
        assert info.status == 1 and n == -1.0, args
        assert _launches(q) == n0, "a refused call launched kernels"
    # the valid handles still work after the refusals
    info = QOP_info_t()
    assert fn(C.byref(info), fla, 0.05, hout, hin, 0) > 0 and info.status == 0
    assert q.lattice_use(lb) == 0
    q.destroy_L(fla_b)
    q.destroy_V(vb)
    assert q.lattice_use(0) == 0
    for h in (hin, hout):
        q.destroy_V(h)
    q.destroy_L(fla)


def test_noalloc_rejects_lattices_beyond_its_scratch():
    L = (16, 16, 16, 40)                             # 81920 sites per parity > 65536
    V = int(np.prod(L))
    q = gpu_lattice(L, "D")
    fn = _fn(q)
    fat = [np.zeros((V, 3, 3, 2)) for _ in range(4)]
    fla = q.create_L_from_raw(fat, fat)
    src = np.zeros((V, 3, 2))
    hin, hout = q.create_V(src), q.create_V(src)
    info = QOP_info_t()
    n = fn(C.byref(info), fla, 0.1, hout, hin, 0)
    assert info.status == 1 and n == -1.0
    for h in (hin, hout):
        q.destroy_V(h)
    q.destroy_L(fla)
