// eom.cu -- EOM-EE-CCSD singlet excitation energies (PROGRAM VEE,
// vee/doeomee_david.F) on the device.
//
// The reference builds the similarity-transformed Hamiltonian Hbar and, per
// irrep, runs a Davidson iteration whose trial products are Hbar times the
// trial vectors (HBARXC) from a Tamm-Dancoff guess (NEWGES), with NEXTDAV
// extrapolating the subspace (vee/doeomee_david.F:99-300).  Here the singlet
// EOM-CCSD spectrum is obtained from the CC Jacobian: with r(T) = Z(T) - D o T
// the closed-shell residual in the pair-symmetric spin-adapted amplitudes,
// J = dr/dT on that subspace is the singlet block of Hbar - E_CC over single
// and double excitations.  Its transpose has the same eigenvalues (the left
// eigenvectors), and its products are exactly what the Lambda code already
// computes: a reverse replay of the residual pass recorded at the converged
// amplitudes gives (dZ/dT)^T x.  So
//     sigma(x) = P[(dZ/dT)^T x] - D o x,   P: the pair symmetriser,
// for x in the pair-symmetric space of irrep h (amplitudes only on the
// excitations whose orbital irreps multiply to h), and a Davidson iteration on
// the device -- trial vectors and products as rows of two device matrices,
// the subspace matrix V S^T grown by one row and column per new vector --
// finds the lowest roots.
// The subspace eigenproblem (a few tens of rows, non-symmetric) is solved on
// the host: Householder reduction to Hessenberg form, complex shifted QR
// with Wilkinson shifts for the eigenvalues, inverse iteration for the
// eigenvector of each selected root (Golub & Van Loan, Matrix Computations,
// 4th ed., sections 7.4-7.6).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <vector>

#include "eig_small.h"
#include "engine.cuh"

namespace acesb200 {

namespace {

using small::cplx;
using small::eig_values;
using small::eig_vector;

// sigma = (g1 - (e_i - e_a) x1, P[g2] - (e_i + e_j - e_a - e_b) x2) on the
// excitations of irrep h, zero elsewhere; g2 already pair-symmetrised (out may
// be g: each element is read before it is written by the same thread)
__global__ void k_eom_combine(double *out, const double *g,
                              const double *__restrict__ x, const double *__restrict__ eo,
                              const double *__restrict__ ev, const int *__restrict__ irr_o,
                              const int *__restrict__ irr_v, int h, int o, int v,
                              long long len) {
  const long long ov = (long long)o * v;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < len;
       n += (long long)gridDim.x * blockDim.x) {
    double d;
    int sym;
    if (n < ov) {
      const int i = (int)(n / v), a = (int)(n % v);
      d = eo[i] - ev[a];
      sym = irr_o[i] ^ irr_v[a];
    } else {
      long long r = n - ov;
      const int b = (int)(r % v); r /= v;
      const int a = (int)(r % v); r /= v;
      const int j = (int)(r % o);
      const int i = (int)(r / o);
      d = eo[i] + eo[j] - ev[a] - ev[b];
      sym = irr_o[i] ^ irr_o[j] ^ irr_v[a] ^ irr_v[b];
    }
    out[n] = sym == h ? g[n] - d * x[n] : 0.0;
  }
}

// Davidson correction: d = res / (omega - diag), diag = -D (the orbital-energy
// differences), small denominators clamped to 1e-2; irrep h only
__global__ void k_eom_precond(double *__restrict__ dvec, const double *__restrict__ res,
                              double omega, const double *__restrict__ eo,
                              const double *__restrict__ ev, const int *__restrict__ irr_o,
                              const int *__restrict__ irr_v, int h, int o, int v,
                              long long len) {
  const long long ov = (long long)o * v;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < len;
       n += (long long)gridDim.x * blockDim.x) {
    double dg;
    int sym;
    if (n < ov) {
      const int i = (int)(n / v), a = (int)(n % v);
      dg = ev[a] - eo[i];
      sym = irr_o[i] ^ irr_v[a];
    } else {
      long long r = n - ov;
      const int b = (int)(r % v); r /= v;
      const int a = (int)(r % v); r /= v;
      const int j = (int)(r % o);
      const int i = (int)(r / o);
      dg = ev[a] + ev[b] - eo[i] - eo[j];
      sym = irr_o[i] ^ irr_o[j] ^ irr_v[a] ^ irr_v[b];
    }
    double den = omega - dg;
    if (std::fabs(den) < 1e-2) den = 1e-2;
    dvec[n] = sym == h ? res[n] / den : 0.0;
  }
}

// c[r] = alpha sum_n A[r * lda + n] y[n] for r < m (m <= kMaxRows): y is read
// once, each row once; every block owns chunks of 1024 elements (4 per
// thread), a warp sums its lanes' products per row and lane 0 adds the sum to
// the warp's shared slot (fixed order: deterministic), and one block of the
// second kernel sums the blocks' partials in block order.
constexpr int kMaxRows = 64, kDotBlocks = 592;
__global__ void __launch_bounds__(256)
    k_multidot(double *__restrict__ part, const double *__restrict__ A, long long lda,
               const double *__restrict__ y, long long len, int m) {
  __shared__ double sh[kMaxRows][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
    for (int r = 0; r < m; ++r) sh[r][wid] = 0.0;
  const long long nchunk = (len + 1023) / 1024;
  for (long long c = blockIdx.x; c < nchunk; c += gridDim.x) {
    const long long n0 = c * 1024 + threadIdx.x;
    double yv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) yv[u] = n0 + 256 * u < len ? y[n0 + 256 * u] : 0.0;
    for (int r = 0; r < m; ++r) {
      const double *a = A + (long long)r * lda;
      double s = 0.0;
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (n0 + 256 * u < len) s += a[n0 + 256 * u] * yv[u];
      for (int off = 16; off; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
      if (lane == 0) sh[r][wid] += s;
    }
  }
  __syncthreads();
  for (int r = threadIdx.x; r < m; r += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += sh[r][w];
    part[(long long)blockIdx.x * kMaxRows + r] = s;
  }
}

__global__ void k_multidot_final(double *__restrict__ c, const double *__restrict__ part, int m,
                                 double alpha) {
  const int r = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < kDotBlocks; b += 32) s += part[(long long)b * kMaxRows + r];
  for (int off = 16; off; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if (threadIdx.x == 0) c[r] = alpha * s;
}

unsigned grid_for(long long n) {
  long long nb = (n + 255) / 256;
  if (nb > 148 * 16) nb = 148 * 16;
  return (unsigned)std::max(1LL, nb);
}

}  // namespace

// sigma = P (dZ/dT)^T x - D o x on irrep h (the tape holds the converged pass)
int CCEngine::eom_sigma(const double *x, double *out, int h, const int *d_irr_o,
                        const int *d_irr_v) {
  const long long ov = (long long)o * v, len = ov + (long long)o * o * v * v;
  const long long O = o, V = v;
  zero_adjoints();
  double *z1b = adj(Z1.p), *z2b = adj(Z2.p);
  if (!z1b || !z2b) return ACES_ERR_NOMEM;
  launch_axpy(z1b, x, 1.0, ov, st);
  launch_axpy(z2b, x + ov, 1.0, len - ov, st);
  // the ladder couples occupied pairs of irrep g ^ h with virtual pairs of
  // irrep g for a vector of irrep h
  ladder_sym = h;
  const int bs = backward();
  ladder_sym = 0;
  ACES_TRY(bs);
  const double *g = adj(X.p);
  // pair symmetriser on the doubles: out2 = (g2 + g2^T) / 2, g2^T[i,j,a,b] = g2[j,i,b,a]
  const long long s2[4] = {O * V * V, V * V, V, 1};
  ACES_CUDA(cudaMemcpyAsync(out, g, ov * 8, cudaMemcpyDeviceToDevice, st));
  PermSpec ps;
  ps.n[0] = o; ps.n[1] = o; ps.n[2] = v; ps.n[3] = v;
  ps.nterms = 2;
  ps.beta = 0.0;
  ps.t[0] = PermTerm{g + ov, 0.5, {s2[0], s2[1], s2[2], s2[3]}};
  ps.t[1] = PermTerm{g + ov, 0.5, {s2[1], s2[0], s2[3], s2[2]}};
  ACES_TRY(permute(out + ov, ps, st));
  k_eom_combine<<<grid_for(len), 256, 0, st>>>(out, out, x, eo.p, ev.p, d_irr_o, d_irr_v, h, o,
                                               v, len);
  count_launch();
  ACES_CUDA(cudaGetLastError());
  return ACES_OK;
}

}  // namespace acesb200

using namespace acesb200;

extern "C" int xvee_run(aces_eom_config *cfg) {
  if (!cfg) return ACES_ERR_ARG;
  State &stt = state();
  std::lock_guard<std::recursive_mutex> lk(stt.mu);
  CCEngine *Ep = engine_instance(false);
  if (!Ep || !Ep->have_amplitudes) {
    set_error("xvee_run: no converged CC amplitudes (run xvcc_run first)");
    return ACES_ERR_ARG;
  }
  CCEngine &E = *Ep;
  const int nirrep = stt.sym.nirrep;
  if (cfg->eom_maxcyc < 1 || cfg->eom_conv < 1 || cfg->eom_conv > 12 || cfg->max_subspace < 0) {
    set_error("xvee_run: eom_maxcyc >= 1, eom_conv 1..12 and max_subspace >= 0 required");
    return ACES_ERR_ARG;
  }
  for (int h = 0; h < 8; ++h)
    if (cfg->nroots[h] < 0 || cfg->nroots[h] > 8 || (h >= nirrep && cfg->nroots[h] > 0)) {
      set_error("xvee_run: nroots[%d] = %d (0..8 roots in irreps 1..%d)", h, cfg->nroots[h],
                nirrep);
      return ACES_ERR_ARG;
    }
  if (cfg->precision != ACES_PREC_FP64 && cfg->precision != ACES_PREC_BF16X3) return ACES_ERR_ARG;
  E.prec = cfg->precision;
  const int o = E.o, v = E.v;
  const long long ov = (long long)o * v, len = ov + (long long)o * o * v * v;
  const double tol = std::pow(10.0, -cfg->eom_conv);
  const int maxdim = cfg->max_subspace > 0 ? cfg->max_subspace : 40;
  auto t_start = std::chrono::steady_clock::now();
  // the converged residual pass on the tape; its reverse replay is (dZ/dT)^T x
  ACES_TRY(E.record_residual(false));
  DBuf Vm, Sm, xr, sr, rv, dv, cdev, irrbuf, dpart;
  struct Release {
    CCEngine &E;
    std::vector<DBuf *> b;
    ~Release() {
      cudaStreamSynchronize(E.st);
      for (DBuf *p : b)
        if (p->p) dev_free(p->p);
    }
  } release{E, {&Vm, &Sm, &xr, &sr, &rv, &dv, &cdev, &irrbuf, &dpart}};
  ACES_TRY(E.alloc(Vm, (size_t)maxdim * len));
  ACES_TRY(E.alloc(Sm, (size_t)maxdim * len));
  ACES_TRY(E.alloc(xr, len));
  ACES_TRY(E.alloc(sr, len));
  ACES_TRY(E.alloc(rv, len));
  ACES_TRY(E.alloc(dv, len));
  ACES_TRY(E.alloc(cdev, (size_t)maxdim * maxdim + 64));
  ACES_TRY(E.alloc(irrbuf, (size_t)(o + v + 1) / 2 + 1));
  ACES_TRY(E.alloc(dpart, (size_t)kDotBlocks * kMaxRows));
  int *d_irr_o = reinterpret_cast<int *>(irrbuf.p), *d_irr_v = d_irr_o + o;
  {
    std::vector<int> irr(E.irr_o);
    irr.insert(irr.end(), E.irr_v.begin(), E.irr_v.end());
    ACES_CUDA(cudaMemcpyAsync(d_irr_o, irr.data(), irr.size() * sizeof(int),
                              cudaMemcpyHostToDevice, E.st));
  }
  std::vector<double> heo(E.eps_h.begin(), E.eps_h.begin() + o),
      hev(E.eps_h.begin() + o, E.eps_h.end());
  auto row = [&](DBuf &M, int k) { return M.p + (size_t)k * len; };
  auto dots = [&](const double *A, int m, const double *y, double alpha, double *c) -> int {
    // c[k] = alpha sum_n A[k*len + n] y[n] for k < m, m <= kMaxRows at a time
    for (int r0 = 0; r0 < m; r0 += kMaxRows) {
      const int mr = std::min(kMaxRows, m - r0);
      k_multidot<<<kDotBlocks, 256, 0, E.st>>>(dpart.p, A + (size_t)r0 * len, len, y, len, mr);
      count_launch();
      k_multidot_final<<<mr, 32, 0, E.st>>>(c + r0, dpart.p, mr, alpha);
      count_launch();
    }
    ACES_CUDA(cudaGetLastError());
    return ACES_OK;
  };
  // out = base + sum_k c[k] M[k] over m rows (c on the device)
  auto combine = [&](double *out, const double *base, DBuf &M, int m, const double *c) {
    const double *b = base;
    for (int k0 = 0; k0 < m; k0 += 25) {
      const int n = std::min(25, m - k0);
      std::vector<const double *> p(n);
      for (int k = 0; k < n; ++k) p[k] = row(M, k0 + k);
      launch_lincomb(out, b, c + k0, p.data(), n, len, E.st);
      b = out;
    }
  };
  auto host_scalar = [&](const double *d) -> double {
    double hval = 0.0;
    cudaMemcpyAsync(&hval, d, 8, cudaMemcpyDeviceToHost, E.st);
    cudaStreamSynchronize(E.st);
    return hval;
  };
  for (int h = 0; h < 8; ++h) {
    for (int r = 0; r < 8; ++r) cfg->omega[h][r] = 0.0;
    cfg->converged[h] = 0;
    cfg->niter[h] = 0;
  }
  int total_sigma = 0;
  bool all_conv = true;
  for (int h = 0; h < nirrep; ++h) {
    const int k = cfg->nroots[h];
    if (k == 0) continue;
    // guesses: singles of irrep h with the smallest orbital-energy gaps
    std::vector<std::pair<double, long long>> cand;
    for (int i = 0; i < o; ++i)
      for (int a = 0; a < v; ++a)
        if ((E.irr_o[i] ^ E.irr_v[a]) == h) cand.push_back({hev[a] - heo[i], (long long)i * v + a});
    std::sort(cand.begin(), cand.end());
    const int ng = (int)std::min<size_t>(cand.size(), (size_t)std::max(2 * k, k + 2));
    if (ng < k || ng > maxdim) {
      set_error("xvee_run: irrep %d has %d single excitations for %d roots (subspace %d)", h + 1,
                (int)cand.size(), k, maxdim);
      return ACES_ERR_ARG;
    }
    int m = 0;
    for (int g = 0; g < ng; ++g) {
      ACES_CUDA(cudaMemsetAsync(row(Vm, m), 0, len * 8, E.st));
      const double one = 1.0;
      ACES_CUDA(cudaMemcpyAsync(row(Vm, m) + cand[g].second, &one, 8, cudaMemcpyHostToDevice,
                                E.st));
      ACES_TRY(E.eom_sigma(row(Vm, m), row(Sm, m), h, d_irr_o, d_irr_v));
      ++total_sigma;
      ++m;
    }
    std::vector<double> w_old(k, 0.0), wsel(k, 0.0);
    // subspace matrix G[i][j] = v_i . s_j, kept on the host (maxdim x maxdim):
    // rows and columns 0..mk-1 are known, each new vector adds its row and
    // column (two passes over the subspace instead of m per iteration)
    std::vector<double> Gh((size_t)maxdim * maxdim, 0.0), colb(maxdim), rowb(maxdim);
    int mk = 0;
    bool conv = false;
    int it;
    for (it = 1; it <= cfg->eom_maxcyc; ++it) {
      for (int j = mk; j < m; ++j) {
        ACES_TRY(dots(Vm.p, m, row(Sm, j), 1.0, cdev.p));             // v_i . s_j
        ACES_TRY(dots(Sm.p, m, row(Vm, j), 1.0, cdev.p + maxdim));    // v_j . s_i
        ACES_CUDA(cudaMemcpyAsync(colb.data(), cdev.p, m * 8, cudaMemcpyDeviceToHost, E.st));
        ACES_CUDA(cudaMemcpyAsync(rowb.data(), cdev.p + maxdim, m * 8, cudaMemcpyDeviceToHost,
                                  E.st));
        ACES_CUDA(cudaStreamSynchronize(E.st));
        for (int i = 0; i < m; ++i) {
          Gh[(size_t)i * maxdim + j] = colb[i];
          Gh[(size_t)j * maxdim + i] = rowb[i];
        }
      }
      mk = m;
      std::vector<double> G((size_t)m * m);
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) G[(size_t)i * m + j] = Gh[(size_t)i * maxdim + j];
      if (int tcs = tc_status_and_clear()) {
        set_error("xvee_run: tensor-core contraction gave up waiting (code %d)", tcs);
        return ACES_ERR_TIMEOUT;
      }
      for (double x : G)
        if (!std::isfinite(x)) {
          set_error("xvee_run: non-finite subspace matrix (irrep %d)", h + 1);
          return ACES_ERR_NAN;
        }
      std::vector<cplx> ev = eig_values(G, m);
      std::vector<double> wr(m);
      for (int q = 0; q < m; ++q) wr[q] = ev[q].real();
      std::sort(wr.begin(), wr.end());
      bool done = true;
      std::vector<std::vector<double>> Y(k);
      for (int r = 0; r < k; ++r) {
        wsel[r] = wr[r];
        Y[r] = eig_vector(G, m, wr[r]);
      }
      std::vector<int> need;
      std::vector<double> rn(k, 0.0);
      for (int r = 0; r < k; ++r) {
        // Ritz vector x = sum y_i v_i, A x = sum y_i s_i, residual A x - w x
        ACES_CUDA(cudaMemcpyAsync(cdev.p, Y[r].data(), m * 8, cudaMemcpyHostToDevice, E.st));
        combine(xr.p, nullptr, Vm, m, cdev.p);
        combine(sr.p, nullptr, Sm, m, cdev.p);
        ACES_CUDA(cudaMemcpyAsync(rv.p, sr.p, len * 8, cudaMemcpyDeviceToDevice, E.st));
        launch_axpy(rv.p, xr.p, -wsel[r], len, E.st);
        ACES_TRY(dots(rv.p, 1, rv.p, 1.0, cdev.p));
        rn[r] = std::sqrt(std::max(0.0, host_scalar(cdev.p)));
        if (rn[r] > tol || std::fabs(wsel[r] - w_old[r]) > tol) {
          done = false;
          if (m < maxdim) {
            k_eom_precond<<<grid_for(len), 256, 0, E.st>>>(dv.p, rv.p, wsel[r], E.eo.p, E.ev.p,
                                                           d_irr_o, d_irr_v, h, o, v, len);
            count_launch();
            ACES_CUDA(cudaGetLastError());
            // Gram-Schmidt against the subspace, twice
            for (int pass = 0; pass < 2; ++pass) {
              ACES_TRY(dots(Vm.p, m, dv.p, -1.0, cdev.p));
              combine(dv.p, dv.p, Vm, m, cdev.p);
            }
            ACES_TRY(dots(dv.p, 1, dv.p, 1.0, cdev.p));
            const double nd = std::sqrt(std::max(0.0, host_scalar(cdev.p)));
            if (nd > 1e-10) {
              ACES_CUDA(cudaMemcpyAsync(row(Vm, m), dv.p, len * 8, cudaMemcpyDeviceToDevice,
                                        E.st));
              launch_scale(row(Vm, m), 1.0 / nd, len, E.st);
              ACES_TRY(E.eom_sigma(row(Vm, m), row(Sm, m), h, d_irr_o, d_irr_v));
              ++total_sigma;
              ++m;
            }
          }
        }
      }
      if (cfg->verbose) {
        printf("  EOM irrep %d iter %3d dim %3d", h + 1, it, m);
        for (int r = 0; r < k; ++r) printf("  w = %.10f |r| = %.2e", wsel[r], rn[r]);
        printf("\n");
      }
      w_old = wsel;
      if (done) {
        conv = true;
        break;
      }
      if (m >= maxdim) {
        // collapse onto the current Ritz vectors (orthonormalised)
        std::vector<double> Yall((size_t)k * m);
        for (int r = 0; r < k; ++r)
          for (int q = 0; q < m; ++q) Yall[(size_t)r * m + q] = Y[r][q];
        DBuf nv;
        ACES_TRY(E.alloc(nv, (size_t)k * len));
        for (int r = 0; r < k; ++r) {
          ACES_CUDA(cudaMemcpyAsync(cdev.p, Yall.data() + (size_t)r * m, m * 8,
                                    cudaMemcpyHostToDevice, E.st));
          combine(nv.p + (size_t)r * len, nullptr, Vm, m, cdev.p);
        }
        ACES_CUDA(cudaMemcpyAsync(Vm.p, nv.p, (size_t)k * len * 8, cudaMemcpyDeviceToDevice,
                                  E.st));
        ACES_CUDA(cudaStreamSynchronize(E.st));
        dev_free(nv.p);
        // Ritz vector r (row r, r >= m) moves to row m, is orthonormalised
        // against rows 0..m-1 and kept unless it was linearly dependent
        m = 0;
        mk = 0;
        for (int r = 0; r < k; ++r) {
          if (m != r)
            ACES_CUDA(cudaMemcpyAsync(row(Vm, m), row(Vm, r), len * 8, cudaMemcpyDeviceToDevice,
                                      E.st));
          for (int pass = 0; pass < 2 && m > 0; ++pass) {
            ACES_TRY(dots(Vm.p, m, row(Vm, m), -1.0, cdev.p));
            combine(row(Vm, m), row(Vm, m), Vm, m, cdev.p);
          }
          ACES_TRY(dots(row(Vm, m), 1, row(Vm, m), 1.0, cdev.p));
          const double nd = std::sqrt(std::max(0.0, host_scalar(cdev.p)));
          if (nd <= 1e-10) continue;
          launch_scale(row(Vm, m), 1.0 / nd, len, E.st);
          ACES_TRY(E.eom_sigma(row(Vm, m), row(Sm, m), h, d_irr_o, d_irr_v));
          ++total_sigma;
          ++m;
        }
      }
    }
    cfg->niter[h] = std::min(it, cfg->eom_maxcyc);
    cfg->converged[h] = conv ? 1 : 0;
    all_conv = all_conv && conv;
    for (int r = 0; r < k; ++r) cfg->omega[h][r] = wsel[r];
  }
  cfg->nsigma = total_sigma;
  cfg->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  std::vector<double> rec(64);
  for (int h = 0; h < 8; ++h)
    for (int r = 0; r < 8; ++r) rec[(size_t)h * 8 + r] = cfg->omega[h][r];
  aces_putrec("EOMEXCIT", 64 * 8, rec.data());
  if (!all_conv) {
    set_error("xvee_run: the EOM Davidson iteration did not converge in %d cycles",
              cfg->eom_maxcyc);
    return ACES_ERR_NOCONV;
  }
  return ACES_OK;
}
