// dense.cu -- host Jacobi eigensolvers for eigCG (dense.h).
#include "dense.h"
#include <algorithm>
#include <cmath>
#include <numeric>

namespace qopb {

// sort eigenpairs ascending: w and the columns of Z
template <typename S>
static void sort_pairs(int n, std::vector<double> &w, std::vector<S> &Z) {
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return w[a] < w[b]; });
  std::vector<double> w2(n);
  std::vector<S> Z2((size_t)n * n);
  for (int j = 0; j < n; j++) {
    w2[j] = w[idx[j]];
    for (int i = 0; i < n; i++) Z2[(size_t)i * n + j] = Z[(size_t)i * n + idx[j]];
  }
  w.swap(w2);
  Z.swap(Z2);
}

void sym_eig(int n, std::vector<double> &A, std::vector<double> &w, std::vector<double> &Z) {
  Z.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) Z[(size_t)i * n + i] = 1.0;
  auto a = [&](int i, int j) -> double & { return A[(size_t)i * n + j]; };
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0, tot = 0;
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) (i == j ? tot : off) += a(i, j) * a(i, j);
    if (off <= 1e-30 * (tot + off) || off == 0.0) break;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) {
        const double apq = a(p, q);
        if (apq == 0.0) continue;
        const double theta = (a(q, q) - a(p, p)) / (2 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
        const double c = 1 / std::sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < n; k++) {   // A <- A G
          const double akp = a(k, p), akq = a(k, q);
          a(k, p) = c * akp - s * akq;
          a(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < n; k++) {   // A <- G^T A
          const double apk = a(p, k), aqk = a(q, k);
          a(p, k) = c * apk - s * aqk;
          a(q, k) = s * apk + c * aqk;
        }
        for (int k = 0; k < n; k++) {   // Z <- Z G
          const double zkp = Z[(size_t)k * n + p], zkq = Z[(size_t)k * n + q];
          Z[(size_t)k * n + p] = c * zkp - s * zkq;
          Z[(size_t)k * n + q] = s * zkp + c * zkq;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; i++) w[i] = a(i, i);
  sort_pairs(n, w, Z);
}

void herm_eig(int n, std::vector<zc> &A, std::vector<double> &w, std::vector<zc> &Z) {
  Z.assign((size_t)n * n, zc(0, 0));
  for (int i = 0; i < n; i++) Z[(size_t)i * n + i] = 1.0;
  auto a = [&](int i, int j) -> zc & { return A[(size_t)i * n + j]; };
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0, tot = 0;
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) (i == j ? tot : off) += std::norm(a(i, j));
    if (off <= 1e-30 * (tot + off) || off == 0.0) break;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) {
        const zc apq = a(p, q);
        const double r = std::abs(apq);
        if (r == 0.0) continue;
        // unitary rotation in the (p, q) plane that zeroes a(p, q):
        // phase e = apq / |apq| makes the 2x2 block real symmetric
        const zc e = apq / r;
        const double theta = (a(q, q).real() - a(p, p).real()) / (2 * r);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
        const double c = 1 / std::sqrt(t * t + 1), s = t * c;
        // G = [[c, s e], [-s conj(e), c]] acting on columns p, q
        const zc gpq = s * e, gqp = -s * std::conj(e);
        for (int k = 0; k < n; k++) {   // A <- A G
          const zc akp = a(k, p), akq = a(k, q);
          a(k, p) = akp * c + akq * gqp;
          a(k, q) = akp * gpq + akq * c;
        }
        for (int k = 0; k < n; k++) {   // A <- G^+ A
          const zc apk = a(p, k), aqk = a(q, k);
          a(p, k) = c * apk + std::conj(gqp) * aqk;
          a(q, k) = std::conj(gpq) * apk + c * aqk;
        }
        for (int k = 0; k < n; k++) {   // Z <- Z G
          const zc zkp = Z[(size_t)k * n + p], zkq = Z[(size_t)k * n + q];
          Z[(size_t)k * n + p] = zkp * c + zkq * gqp;
          Z[(size_t)k * n + q] = zkp * gpq + zkq * c;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; i++) w[i] = a(i, i).real();
  sort_pairs(n, w, Z);
}

}  // namespace qopb
