"""QOPB_D3_asqtad_ddagd_norm2_noalloc through the C ABI.

This entry point serves callers that cannot allocate device memory where
they apply the operator (a CUDA-graph capture, an application allocator
owning the device memory, allocation-free inner loops).  Its result must
equal the allocating QOP_D3_asqtad_ddagd_norm2 on two calls in a row (the
scratch it reuses keeps the previous call's contents), and lattices beyond
its fixed scratch must be rejected.  Collected last so a failure here cannot
hide other tests; it also passes when run alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import gpu_lattice
from helpers import asqtad_links, site_rel_err
from qopqdp_b200 import lattice as LT
from qopqdp_b200.qop import QOP_info_t

pytestmark = pytest.mark.gpu


def _fn(q):
    f = q.lib.QOPB_D3_asqtad_ddagd_norm2_noalloc
    f.argtypes = [C.POINTER(QOP_info_t), C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_int]
    f.restype = C.c_double
    return f


def test_noalloc_ddagd_norm2_matches_allocating_entry_point():
    L = (8, 8, 8, 8)
    V = int(np.prod(L))
    q = gpu_lattice(L, "D")
    fn = _fn(q)
    fat, lng = asqtad_links(L, 0.3, 7)
    fla = q.create_L_from_raw(fat, lng)
    mass = 0.05
    for eo in (0, 1):
        src = LT.gaussian_vector(L, 200 + eo)
        hin = q.create_V(src)
        href = q.create_V(np.zeros_like(src))
        n_ref = q.ddagd_norm2(fla, mass, href, hin, eo)
        ref = q.extract_V(href, V)
        for call in range(2):                       # scratch reused between calls
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
