// dense.h -- small dense eigenproblems on the host (eigCG's Rayleigh-Ritz
// steps: real symmetric tridiagonal-window matrices of order <= eigcg_m and
// complex Hermitian matrices of order <= eigcg_l).  Cyclic Jacobi rotations
// in FP64; eigenvalues ascending, eigenvectors in the columns of Z
// (row-major n x n: Z[i * n + j] is component i of eigenvector j).
#pragma once
#include <complex>
#include <vector>

namespace qopb {

typedef std::complex<double> zc;

// A (n x n, symmetric, row-major) is overwritten
void sym_eig(int n, std::vector<double> &A, std::vector<double> &w, std::vector<double> &Z);
// A (n x n, Hermitian, row-major) is overwritten
void herm_eig(int n, std::vector<zc> &A, std::vector<double> &w, std::vector<zc> &Z);

}  // namespace qopb
