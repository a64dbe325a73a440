"""Seeded synthetic inputs in the reference raw layout.

Gauge links U = exp(i eps H) with H = sum_a h_a lambda_a / 2 traceless
Hermitian, h_a ~ N(0, 1) (8 Gell-Mann coefficients per link); sources are
Gaussian with unit variance per real component.  Random numbers come from
numpy's Philox generator keyed by the seed, drawn in raw site order, so a
(lattice, seed) pair always gives the same field on any host.  The
reference's own generator (QLA gaussian) is not available, so these fields
stand in for examples/test_common.c get_random_links / gaussian sources.

Raw order: even sites first, then odd; within a parity lex/2 with x[0]
slowest and x[3] fastest (lib/layout_user.c:237-258).
"""
import numpy as np

# examples/asqtad_invert_bench.c:119-124 (the only asqtad coefficient set the
# reference ships): one_link, three, five, seven, lepage, naik
ASQTAD_BENCH_COEFFS = (1.0, 0.1, 0.1, 0.1, 0.1, 0.1)

# examples/asqtad_test.c:275-281: t antiperiodic, staggered sign masks
BENCH_R0 = (0, 0, 0, 0)
BENCH_BC = (1, 1, 1, -1)
BENCH_SIGNMASK = (0, 1, 3, 7)


def hisq_bench_coeffs():
    """examples/hisq_invert_bench.c:107-125 (U(3), analytic, n_naiks = 1)."""
    from .qop import QOP_hisq_coeffs_t, QOP_UNITARIZE_U3, QOP_UNITARIZE_ANALYTIC
    c = QOP_hisq_coeffs_t()
    c.n_naiks = 1
    c.ugroup = QOP_UNITARIZE_U3
    c.umethod = QOP_UNITARIZE_ANALYTIC
    c.fat7_one_link, c.fat7_three_staple, c.fat7_five_staple, c.fat7_seven_staple = 1.0, 0.1, 0.1, 0.1
    c.asqtad_one_link, c.asqtad_three_staple, c.asqtad_five_staple = 1.0, 0.1, 0.1
    c.asqtad_seven_staple, c.asqtad_lepage, c.asqtad_naik = 0.1, 0.1, 0.1
    return c


def hisq_coeff_vector(c, force_filter=5e-5):
    """18-double layout used by the oracle's HISQ routines: the 13
    coefficients, then use_fat7_lepage, reunit_allow_svd, svd_rel_error,
    svd_abs_error (QOP_hisq_links_set_opts defaults) and the force filter
    (QOP_hisq_force_set_opts default, lib/hisq_force.c:4-9)."""
    return np.array([c.fat7_one_link, c.fat7_three_staple, c.fat7_five_staple, c.fat7_seven_staple, c.fat7_lepage,
                     c.asqtad_one_link, c.asqtad_three_staple, c.asqtad_five_staple, c.asqtad_seven_staple,
                     c.asqtad_lepage, c.asqtad_naik, c.difference_one_link, c.difference_naik,
                     0.0, 1.0, 1e-8, 1e-8, force_filter], dtype=np.float64)


def volume(L):
    return int(np.prod(L))


def raw_coords(L):
    """(V, 4) int array: coordinates of each raw site index."""
    L = tuple(int(x) for x in L)
    V = volume(L)
    lex = np.arange(V, dtype=np.int64)
    x = np.empty((V, 4), dtype=np.int64)
    t = lex.copy()
    for i in range(3, -1, -1):
        x[:, i] = t % L[i]
        t //= L[i]
    par = x.sum(axis=1) & 1
    raw = np.where(par == 0, lex // 2, (lex + V) // 2)
    out = np.empty_like(x)
    out[raw] = x
    return out


def raw_index(L, x):
    x = np.asarray(x, dtype=np.int64)
    lex = ((x[..., 0] * L[1] + x[..., 1]) * L[2] + x[..., 2]) * L[3] + x[..., 3]
    V = volume(L)
    return np.where(x.sum(axis=-1) % 2 == 0, lex // 2, (lex + V) // 2)


def _gell_mann_half():
    l = np.zeros((8, 3, 3), dtype=np.complex128)
    l[0, 0, 1] = l[0, 1, 0] = 1
    l[1, 0, 1], l[1, 1, 0] = -1j, 1j
    l[2, 0, 0], l[2, 1, 1] = 1, -1
    l[3, 0, 2] = l[3, 2, 0] = 1
    l[4, 0, 2], l[4, 2, 0] = -1j, 1j
    l[5, 1, 2] = l[5, 2, 1] = 1
    l[6, 1, 2], l[6, 2, 1] = -1j, 1j
    l[7] = np.diag([1, 1, -2]) / np.sqrt(3)
    return l / 2


def random_gauge(L, eps, seed, device="cpu"):
    """4 float64 arrays (V, 3, 3, 2): U_mu = exp(i eps H_mu(x)) in raw order.

    device: 'cpu' or a CUDA device for the matrix exponential (torch is used
    only as a batched expm; the Gaussians always come from numpy Philox).
    """
    import torch
    V = volume(L)
    rng = np.random.Generator(np.random.Philox(key=int(seed)))
    T = _gell_mann_half()
    out = []
    for mu in range(4):
        h = rng.standard_normal((V, 8))
        H = np.einsum("va,aij->vij", h, T)
        A = torch.from_numpy(1j * eps * H).to(device)
        U = torch.linalg.matrix_exp(A).cpu().numpy()
        del A
        out.append(np.ascontiguousarray(np.stack([U.real, U.imag], axis=-1)))
    return out


def gaussian_vector(L, seed, dtype=np.float64):
    """(V, 3, 2) Gaussian source, unit variance per real component."""
    V = volume(L)
    rng = np.random.Generator(np.random.Philox(key=int(seed) + 0x5EED))
    return rng.standard_normal((V, 3, 2)).astype(dtype)


def parity_mask(L):
    """(V,) bool: True on even sites (the first V/2 raw indices)."""
    V = volume(L)
    m = np.zeros(V, dtype=bool)
    m[: V // 2] = True
    return m


def to_complex(a):
    a = np.asarray(a, dtype=np.float64)
    return a[..., 0] + 1j * a[..., 1]


def from_complex(z, dtype=np.float64):
    return np.ascontiguousarray(np.stack([z.real, z.imag], axis=-1)).astype(dtype)
