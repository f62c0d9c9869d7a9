// adjoint.cuh -- reverse-mode (adjoint) replay of the CCSD residual.
//
// The Lambda equations are the adjoint of the CC amplitude equations
// (lambda/README: the left-hand eigenvector of the similarity-transformed
// Hamiltonian), and the one-particle density is the derivative of the CC
// Lagrangian with respect to the Fock matrix.  Both need products with the
// transpose of the residual's Jacobian.  The engine records, during one
// forward residual pass at fixed amplitudes, every operation that touches an
// amplitude-dependent (or Fock-dependent) buffer; the backward pass walks the
// tape in reverse and applies each operation's adjoint with dedicated
// kernels (transposed contractions, scatter-add resorts, the tau adjoint).
#pragma once
#include <vector>

#include "gemm.cuh"
#include "kernels.cuh"

namespace acesb200 {

struct TapeOp {
  enum Kind { GEMM, PERM, COPY, TAU, LADDER } kind;
  // GEMM: C(view) = alpha * A B^T + beta * C
  int M = 0, N = 0, K = 0;
  double alpha = 0, beta = 0;
  const double *A = nullptr, *B = nullptr;
  long long lda = 0, ldb = 0;
  CView C{};
  bool a_act = false, b_act = false, c_act = false;
  // PERM: out = beta*out + sum_t alpha_t perm_t(src_t)
  double *out = nullptr;
  PermSpec spec{};
  bool t_act[4] = {false, false, false, false};
  // COPY: dst <- src (count doubles)
  // LADDER: dst[ij,ab] += sum_cd <ab|cd> src[ij,cd] (the packed pp ladder)
  double *dst = nullptr;
  const double *src = nullptr;
  size_t count = 0;
  // TAU: tau = t2 + c t1 (x) t1 over [o,o,v,v]
  double *tau = nullptr;
  const double *t2 = nullptr, *t1 = nullptr;
  double c = 0;
};

// adjoint kernels
// dense[m*N + n] = scale * C(view)(m, n)
void launch_view_gather(double *dense, const CView &C, int M, int N, double scale,
                        cudaStream_t st);
// C(view)(m,n) = value over all (m,n) (beta == 0 adjoint) or C *= value
void launch_view_scale(const CView &C, int M, int N, double value, cudaStream_t st);
// src_bar[addr_t(idx)] += alpha * out_bar[idx]  (adjoint of one permute term)
void launch_perm_scatter_add(double *src_bar, const double *out_bar, const PermTerm &t,
                             const int n[4], cudaStream_t st);
// y += a * x over n elements
void launch_axpy(double *y, const double *x, double a, long long n, cudaStream_t st);
void launch_scale(double *y, double a, long long n, cudaStream_t st);
// tau adjoint: t2_bar += tau_bar; t1_bar += c * (contractions with t1)
void launch_tau_adjoint(double *t2_bar, double *t1_bar, const double *tau_bar,
                        const double *t1, double c, int o, int v, cudaStream_t st);

}  // namespace acesb200
