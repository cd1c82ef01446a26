// eig.hpp -- dense symmetric eigen-decompositions on the host (plain C++,
// no CUDA): the per-axis factorizations of the fast-diagonalization Poisson
// solve.  Row-major matrices; eigenvectors are the columns of V.
#pragma once
#include <cmath>
#include <vector>

namespace eig {

// symmetric eigen-decomposition by cyclic Jacobi: A (n x n, row-major) ->
// eigenvalues w and eigenvectors as the columns of V (row-major)
inline void jacobi_eigen(std::vector<double> A, int n, std::vector<double>& w, std::vector<double>& V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) V[(size_t)i * n + i] = 1.0;
  double tot = 0.0;
  for (double v : A) tot += v * v;
  for (int sweep = 0; sweep < 60; sweep++) {
    double off = 0.0;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) off += A[(size_t)p * n + q] * A[(size_t)p * n + q];
    if (off <= 1e-32 * tot) break;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) {
        const double apq = A[(size_t)p * n + q];
        if (apq == 0.0) continue;
        const double tau = (A[(size_t)q * n + q] - A[(size_t)p * n + p]) / (2.0 * apq);
        const double t = (tau >= 0.0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
        const double c = 1.0 / std::sqrt(1.0 + t * t), sn = t * c;
        for (int k = 0; k < n; k++) {  // A <- A J
          const double akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
          A[(size_t)k * n + p] = c * akp - sn * akq;
          A[(size_t)k * n + q] = sn * akp + c * akq;
        }
        for (int k = 0; k < n; k++) {  // A <- J^T A
          const double apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
          A[(size_t)p * n + k] = c * apk - sn * aqk;
          A[(size_t)q * n + k] = sn * apk + c * aqk;
        }
        for (int k = 0; k < n; k++) {  // V <- V J
          const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
          V[(size_t)k * n + p] = c * vkp - sn * vkq;
          V[(size_t)k * n + q] = sn * vkp + c * vkq;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; i++) w[i] = A[(size_t)i * n + i];
}

// symmetric tridiagonal eigen-decomposition by the implicit QL iteration
// with Wilkinson shifts (Bowdler, Martin, Reinsch & Wilkinson, Numer. Math.
// 11, 1968): diagonal d, off-diagonal e (e[i] couples i and i+1) ->
// eigenvalues in d, eigenvectors as the columns of V (row-major); false
// when an eigenvalue needs more than 60 sweeps
inline bool tridiag_ql(std::vector<double> d, std::vector<double> e, int n, std::vector<double>& w, std::vector<double>& V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) V[(size_t)i * n + i] = 1.0;
  e.resize(n, 0.0);
  e[n - 1] = 0.0;
  for (int l = 0; l < n; l++) {
    for (int iter = 0;; iter++) {
      int m = l;
      for (; m < n - 1; m++) {
        const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= 1e-16 * dd) break;
      }
      if (m == l) break;
      if (iter >= 60) return false;
      // shift from the leading 2x2 block's eigenvalue closer to d[l]
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? r : -r));
      double sn = 1.0, c = 1.0, p = 0.0;
      int i = m - 1;
      bool split = false;
      for (; i >= l; i--) {  // chase the bulge from the bottom of the block up
        const double f = sn * e[i], b = c * e[i];
        r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {  // the block splits: deflate and restart
          d[i + 1] -= p;
          e[m] = 0.0;
          split = true;
          break;
        }
        sn = f / r;
        c = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * sn + 2.0 * c * b;
        p = sn * r;
        d[i + 1] = g + p;
        g = c * r - b;
        for (int k = 0; k < n; k++) {  // accumulate the rotation in the vectors
          const double vi = V[(size_t)k * n + i], vi1 = V[(size_t)k * n + i + 1];
          V[(size_t)k * n + i + 1] = sn * vi + c * vi1;
          V[(size_t)k * n + i] = c * vi - sn * vi1;
        }
      }
      if (split) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  w = d;
  return true;
}

// Householder reduction of a symmetric matrix to tridiagonal form, A =
// Q T Q^T (Golub & Van Loan, Alg. 8.3.1): diagonal d and off-diagonal e of
// T, Q row-major.  Reflector k zeroes column k below the subdiagonal, applied
// to the trailing block as the symmetric rank-2 update A -= v w^T + w v^T.
inline void householder_tridiag(std::vector<double> A, int n, std::vector<double>& d, std::vector<double>& e,
                         std::vector<double>& Q) {
  Q.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) Q[(size_t)i * n + i] = 1.0;
  std::vector<double> v(n), p(n), w(n);
  for (int k = 0; k + 2 < n; k++) {
    const int m = n - k - 1;  // length of the column part below the diagonal
    double nrm = 0.0;
    for (int i = 0; i < m; i++) nrm += A[(size_t)(k + 1 + i) * n + k] * A[(size_t)(k + 1 + i) * n + k];
    nrm = std::sqrt(nrm);
    if (nrm == 0.0) continue;
    const double x0 = A[(size_t)(k + 1) * n + k];
    const double alpha = x0 >= 0.0 ? -nrm : nrm;
    for (int i = 0; i < m; i++) v[i] = A[(size_t)(k + 1 + i) * n + k];
    v[0] -= alpha;
    double vn = 0.0;
    for (int i = 0; i < m; i++) vn += v[i] * v[i];
    vn = std::sqrt(vn);
    if (vn == 0.0) continue;
    for (int i = 0; i < m; i++) v[i] /= vn;
    // p = 2 A22 v, w = p - (v.p) v
    double vp = 0.0;
    for (int i = 0; i < m; i++) {
      double acc = 0.0;
      const double* row = &A[(size_t)(k + 1 + i) * n + (k + 1)];
      for (int j = 0; j < m; j++) acc += row[j] * v[j];
      p[i] = 2.0 * acc;
      vp += v[i] * p[i];
    }
    for (int i = 0; i < m; i++) w[i] = p[i] - vp * v[i];
    for (int i = 0; i < m; i++) {
      double* row = &A[(size_t)(k + 1 + i) * n + (k + 1)];
      for (int j = 0; j < m; j++) row[j] -= v[i] * w[j] + w[i] * v[j];
    }
    A[(size_t)(k + 1) * n + k] = A[(size_t)k * n + k + 1] = alpha;
    for (int i = 1; i < m; i++) A[(size_t)(k + 1 + i) * n + k] = A[(size_t)k * n + k + 1 + i] = 0.0;
    // Q <- Q H: Q[:, k+1:] -= 2 (Q[:, k+1:] v) v^T
    for (int r = 0; r < n; r++) {
      double* row = &Q[(size_t)r * n + (k + 1)];
      double acc = 0.0;
      for (int j = 0; j < m; j++) acc += row[j] * v[j];
      acc *= 2.0;
      for (int j = 0; j < m; j++) row[j] -= acc * v[j];
    }
  }
  d.assign(n, 0.0);
  e.assign(n, 0.0);
  for (int i = 0; i < n; i++) d[i] = A[(size_t)i * n + i];
  for (int i = 0; i + 1 < n; i++) e[i] = A[(size_t)i * n + i + 1];
}

// symmetric eigen-decomposition of a full matrix: Householder reduction,
// then the QL iteration on T, eigenvectors Q V_T; cyclic Jacobi if the QL
// iteration does not converge
inline void symmetric_eigen(const std::vector<double>& A, int n, std::vector<double>& w, std::vector<double>& V) {
  std::vector<double> d, e, Q, VT;
  householder_tridiag(A, n, d, e, Q);
  if (!tridiag_ql(d, e, n, w, VT)) {
    jacobi_eigen(A, n, w, V);
    return;
  }
  V.assign((size_t)n * n, 0.0);
  for (int r = 0; r < n; r++)
    for (int k = 0; k < n; k++) {
      const double q = Q[(size_t)r * n + k];
      if (q == 0.0) continue;
      const double* vt = &VT[(size_t)k * n];
      double* out = &V[(size_t)r * n];
      for (int c = 0; c < n; c++) out[c] += q * vt[c];
    }
}

}  // namespace eig
