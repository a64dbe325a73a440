"""The host eigensolvers of eigCG (qopqdp_b200/csrc/dense.cu: cyclic Jacobi
for real symmetric and complex Hermitian matrices) against numpy.linalg.eigh
on random and degenerate matrices.  dense.cu is host code; the test builds
it with a small C wrapper into a throwaway shared library (no GPU)."""
import ctypes as C
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DENSE = os.path.join(ROOT, "qopqdp_b200", "csrc", "dense.cu")

WRAP = r"""
#include "dense.h"
#include <vector>
using namespace qopb;
extern "C" void t_sym_eig(int n, double *a, double *w, double *z) {
  std::vector<double> A(a, a + (size_t)n * n), W, Z;
  sym_eig(n, A, W, Z);
  for (int i = 0; i < n; i++) w[i] = W[i];
  for (size_t k = 0; k < (size_t)n * n; k++) z[k] = Z[k];
}
extern "C" void t_herm_eig(int n, double *a, double *w, double *z) {
  std::vector<zc> A((size_t)n * n), Z;
  std::vector<double> W;
  for (size_t k = 0; k < (size_t)n * n; k++) A[k] = zc(a[2 * k], a[2 * k + 1]);
  herm_eig(n, A, W, Z);
  for (int i = 0; i < n; i++) w[i] = W[i];
  for (size_t k = 0; k < (size_t)n * n; k++) { z[2 * k] = Z[k].real(); z[2 * k + 1] = Z[k].imag(); }
}
"""


@pytest.fixture(scope="module")
def lib():
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no g++")
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "wrap.cpp"), "w") as f:
        f.write(WRAP)
    # dense.cu holds host code only: compile it as C++
    shutil.copy(DENSE, os.path.join(d, "dense.cpp"))
    so = os.path.join(d, "libdense.so")
    subprocess.run([cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-I", os.path.dirname(DENSE),
                    os.path.join(d, "dense.cpp"), os.path.join(d, "wrap.cpp"), "-o", so], check=True)
    lib = C.CDLL(so)
    dp = C.POINTER(C.c_double)
    for name in ("t_sym_eig", "t_herm_eig"):
        getattr(lib, name).argtypes = [C.c_int, dp, dp, dp]
    yield lib
    shutil.rmtree(d, ignore_errors=True)


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@pytest.mark.parametrize("n", [1, 2, 7, 40])
def test_sym_eig_matches_numpy(lib, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n))
    a = np.ascontiguousarray(a + a.T)
    w, z = np.zeros(n), np.zeros((n, n))
    lib.t_sym_eig(n, _p(a.copy()), _p(w), _p(z))
    assert np.allclose(w, np.linalg.eigvalsh(a), rtol=0, atol=1e-12 * max(1, np.abs(a).max()))
    assert np.all(np.diff(w) >= 0)
    assert np.allclose(z.T @ z, np.eye(n), atol=1e-12)
    assert np.allclose(a @ z, z * w, atol=1e-10 * max(1, np.abs(a).max()))


@pytest.mark.parametrize("n", [1, 3, 16, 60])
def test_herm_eig_matches_numpy(lib, n):
    rng = np.random.default_rng(100 + n)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    a = np.ascontiguousarray(a + a.conj().T)
    w, z = np.zeros(n), np.zeros((n, n, 2))
    lib.t_herm_eig(n, _p(a.view(np.float64).copy()), _p(w), _p(z))
    zc = z[..., 0] + 1j * z[..., 1]
    assert np.allclose(w, np.linalg.eigvalsh(a), rtol=0, atol=1e-11 * max(1, np.abs(a).max()))
    assert np.allclose(zc.conj().T @ zc, np.eye(n), atol=1e-11)
    assert np.allclose(a @ zc, zc * w, atol=1e-9 * max(1, np.abs(a).max()))


def test_degenerate_and_diagonal_spectra(lib):
    """Equal eigenvalues (eigCG's windows hold converged duplicates) and an
    already diagonal matrix (no rotation needed)."""
    n = 12
    rng = np.random.default_rng(7)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    lam = np.repeat([1e-4, 0.5, 3.0], 4)
    a = np.ascontiguousarray((q * lam) @ q.conj().T)
    w, z = np.zeros(n), np.zeros((n, n, 2))
    lib.t_herm_eig(n, _p(a.view(np.float64).copy()), _p(w), _p(z))
    assert np.allclose(w, lam, rtol=0, atol=1e-12)
    zc = z[..., 0] + 1j * z[..., 1]
    assert np.allclose(a @ zc, zc * w, atol=1e-11)
    d = np.ascontiguousarray(np.diag([3.0, -1.0, 2.0]))
    w3, z3 = np.zeros(3), np.zeros((3, 3))
    lib.t_sym_eig(3, _p(d.copy()), _p(w3), _p(z3))
    assert np.array_equal(w3, [-1.0, 2.0, 3.0])
    assert np.allclose(np.abs(z3), np.array([[0, 0, 1], [1, 0, 0], [0, 1, 0]]))
