// eig_small.h -- eigenvalues and eigenvectors of small dense real
// non-symmetric matrices (host code; the Davidson subspace of the EOM solver,
// eom.cu).  Householder reduction to upper Hessenberg form, complex explicit
// shifted QR with Wilkinson shifts and deflation for the eigenvalues, and
// inverse iteration for the eigenvector of a chosen real eigenvalue (Golub &
// Van Loan, Matrix Computations, 4th ed., sections 7.4-7.6).  Plain C++ so it
// can be checked on the host without a GPU.
#pragma once
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

namespace acesb200 {
namespace small {

using cplx = std::complex<double>;

// Eigenvalues of the real n x n matrix A (row-major).
inline std::vector<cplx> eig_values(std::vector<double> A, int n) {
  // Householder reduction to upper Hessenberg form (similarity)
  for (int k = 0; k + 2 < n; ++k) {
    double norm = 0.0;
    for (int i = k + 1; i < n; ++i) norm += A[(size_t)i * n + k] * A[(size_t)i * n + k];
    norm = std::sqrt(norm);
    if (norm == 0.0) continue;
    const double x0 = A[(size_t)(k + 1) * n + k];
    const double alpha = x0 >= 0.0 ? -norm : norm;
    std::vector<double> u(n, 0.0);
    for (int i = k + 1; i < n; ++i) u[i] = A[(size_t)i * n + k];
    u[k + 1] -= alpha;
    double un = 0.0;
    for (int i = k + 1; i < n; ++i) un += u[i] * u[i];
    if (un == 0.0) continue;
    // A <- (I - 2uu^T/un) A (I - 2uu^T/un)
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int i = k + 1; i < n; ++i) s += u[i] * A[(size_t)i * n + j];
      s *= 2.0 / un;
      for (int i = k + 1; i < n; ++i) A[(size_t)i * n + j] -= s * u[i];
    }
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int j = k + 1; j < n; ++j) s += A[(size_t)i * n + j] * u[j];
      s *= 2.0 / un;
      for (int j = k + 1; j < n; ++j) A[(size_t)i * n + j] -= s * u[j];
    }
  }
  std::vector<cplx> H((size_t)n * n);
  for (size_t q = 0; q < H.size(); ++q) H[q] = A[q];
  auto h = [&](int i, int j) -> cplx & { return H[(size_t)i * n + j]; };
  std::vector<cplx> ev(n);
  std::vector<cplx> cs(n), sn(n);
  int hi = n - 1, since = 0, total = 0;
  while (hi >= 0) {
    if (hi == 0) {
      ev[0] = h(0, 0);
      break;
    }
    // deflation: the active block is [lo, hi]
    int lo = hi;
    while (lo > 0) {
      const double sub = std::abs(h(lo, lo - 1));
      if (sub <= 1e-15 * (std::abs(h(lo, lo)) + std::abs(h(lo - 1, lo - 1))) || sub < 1e-300) {
        h(lo, lo - 1) = 0.0;
        break;
      }
      --lo;
    }
    if (lo == hi) {
      ev[hi] = h(hi, hi);
      --hi;
      since = 0;
      continue;
    }
    if (++total > 100 * n) {  // no convergence: report the diagonal as it stands
      for (int k = 0; k <= hi; ++k) ev[k] = h(k, k);
      break;
    }
    // Wilkinson shift: the eigenvalue of the trailing 2 x 2 block nearer h(hi,hi);
    // an exceptional shift after 10 sweeps without deflation
    cplx mu;
    if (++since % 11 == 10) {
      mu = h(hi, hi) + std::abs(h(hi, hi - 1));
    } else {
      const cplx a = h(hi - 1, hi - 1), b = h(hi - 1, hi), c = h(hi, hi - 1), d = h(hi, hi);
      const cplx tr2 = 0.5 * (a + d), disc = std::sqrt(0.25 * (a - d) * (a - d) + b * c);
      const cplx m1 = tr2 + disc, m2 = tr2 - disc;
      mu = std::abs(m1 - d) < std::abs(m2 - d) ? m1 : m2;
    }
    // one explicit QR step of the active block: H - mu I = QR, H <- RQ + mu I
    for (int k = lo; k <= hi; ++k) h(k, k) -= mu;
    for (int k = lo; k < hi; ++k) {
      const cplx a = h(k, k), b = h(k + 1, k);
      const double r = std::sqrt(std::norm(a) + std::norm(b));
      const cplx c = r > 0.0 ? a / r : cplx(1.0), s = r > 0.0 ? b / r : cplx(0.0);
      cs[k] = c;
      sn[k] = s;
      for (int j = k; j <= hi; ++j) {
        const cplx t1 = h(k, j), t2 = h(k + 1, j);
        h(k, j) = std::conj(c) * t1 + std::conj(s) * t2;
        h(k + 1, j) = -s * t1 + c * t2;
      }
    }
    for (int k = lo; k < hi; ++k) {
      const cplx c = cs[k], s = sn[k];
      for (int i = lo; i <= std::min(k + 1, hi); ++i) {
        const cplx t1 = h(i, k), t2 = h(i, k + 1);
        h(i, k) = t1 * c + t2 * s;
        h(i, k + 1) = -t1 * std::conj(s) + t2 * std::conj(c);
      }
    }
    for (int k = lo; k <= hi; ++k) h(k, k) += mu;
  }
  return ev;
}

// Solve M y = b in place (row-major n x n, partial pivoting); false if singular.
inline bool lu_solve(std::vector<double> M, int n, std::vector<double> &b) {
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(M[(size_t)i * n + k]) > std::fabs(M[(size_t)p * n + k])) p = i;
    if (M[(size_t)p * n + k] == 0.0) return false;
    if (p != k) {
      for (int j = 0; j < n; ++j) std::swap(M[(size_t)p * n + j], M[(size_t)k * n + j]);
      std::swap(b[p], b[k]);
    }
    for (int i = k + 1; i < n; ++i) {
      const double f = M[(size_t)i * n + k] / M[(size_t)k * n + k];
      if (f == 0.0) continue;
      for (int j = k; j < n; ++j) M[(size_t)i * n + j] -= f * M[(size_t)k * n + j];
      b[i] -= f * b[k];
    }
  }
  for (int k = n - 1; k >= 0; --k) {
    double s = b[k];
    for (int j = k + 1; j < n; ++j) s -= M[(size_t)k * n + j] * b[j];
    b[k] = s / M[(size_t)k * n + k];
  }
  return true;
}

// Right eigenvector of the real matrix G for the (real) eigenvalue lambda, by
// inverse iteration with a slightly perturbed shift.
inline std::vector<double> eig_vector(const std::vector<double> &G, int n, double lambda) {
  std::vector<double> y(n, 1.0 / std::sqrt((double)n));
  const double shift = lambda + 1e-10 * std::max(1.0, std::fabs(lambda));
  std::vector<double> M(G);
  for (int i = 0; i < n; ++i) M[(size_t)i * n + i] -= shift;
  for (int it = 0; it < 4; ++it) {
    if (!lu_solve(M, n, y)) break;
    double nrm = 0.0;
    for (double x : y) nrm += x * x;
    nrm = std::sqrt(nrm);
    if (!(nrm > 0.0) || !std::isfinite(nrm)) break;
    for (double &x : y) x /= nrm;
  }
  return y;
}

}  // namespace small
}  // namespace acesb200
