// xgemm.cu -- the reference's XGEMM boundary (tools/xgemm.F:10-49) on device
// pointers, routed to the engine's contraction kernels.
#include <algorithm>
#include <cctype>

#include "common.cuh"
#include "gemm.cuh"
#include "kernels.cuh"

using namespace acesb200;

namespace {
// dst[r*cols + c] = src[r + c*ld]: column-major (rows x cols) -> row-major
int to_kmajor(double **dst, const double *src, int rows, int cols, long long ld,
              cudaStream_t st) {
  ACES_CUDA(dev_alloc((void **)dst, (size_t)rows * cols * 8 + 8));
  PermSpec s;
  s.n[0] = 1; s.n[1] = 1; s.n[2] = rows; s.n[3] = cols;
  s.nterms = 1;
  s.beta = 0.0;
  s.t[0].src = src;
  s.t[0].alpha = 1.0;
  s.t[0].s[0] = 0; s.t[0].s[1] = 0; s.t[0].s[2] = 1; s.t[0].s[3] = ld;
  return permute(*dst, s, st);
}
}  // namespace

extern "C" int aces_xgemm(char transa, char transb, int m, int n, int k, double alpha,
                          const double *A, int lda, const double *B, int ldb, double beta,
                          double *Cm, int ldc, int precision) {
  char ta = (char)toupper(transa), tb = (char)toupper(transb);
  if ((ta != 'N' && ta != 'T') || (tb != 'N' && tb != 'T') || m < 0 || n < 0 || k < 0) {
    set_error("aces_xgemm: bad arguments");
    return ACES_ERR_ARG;
  }
  if ((long long)m * n == 0) return ACES_OK;  // quick return (tools/xgemm.F)
  if (ldc < (m > 1 ? m : 1)) {
    set_error("aces_xgemm: ldc < m");
    return ACES_ERR_ARG;
  }
  // leading dimensions as DGEMM checks them: op(A) is m x k, op(B) is k x n
  if (lda < std::max(1, ta == 'N' ? m : k) || ldb < std::max(1, tb == 'N' ? k : n)) {
    set_error("aces_xgemm: lda %d or ldb %d below the operand's row count", lda, ldb);
    return ACES_ERR_ARG;
  }
  cudaStream_t st = 0;
  // NT form: Ak[i*K + l] = op(A)(i,l), Bk[j*K + l] = op(B)(l,j)
  const double *Ak = A, *Bk = B;
  long long ldak = lda, ldbk = ldb;
  double *tA = nullptr, *tB = nullptr;
  int status = ACES_OK;
  if (ta == 'N') {  // op(A)(i,l) = A[i + l*lda]
    status = to_kmajor(&tA, A, m, k, lda, st);
    Ak = tA;
    ldak = k;
  }
  if (status == ACES_OK && tb == 'T') {  // op(B)(l,j) = B[j + l*ldb]
    status = to_kmajor(&tB, B, n, k, ldb, st);
    Bk = tB;
    ldbk = k;
  }
  if (status == ACES_OK) {
    CView C = cview_colmajor(Cm, ldc);
    if (precision == ACES_PREC_BF16X3 && k > 0) {
      SplitOperand sa, sb;
      status = split_pack(sa, Ak, ldak, m, k, st);
      if (status == ACES_OK) status = split_pack(sb, Bk, ldbk, n, k, st);
      if (status == ACES_OK) status = gemm_nt_bf16x3(sa, sb, m, n, alpha, beta, C, st);
      cudaStreamSynchronize(st);
      if (sa.hi) dev_free(sa.hi);
      if (sb.hi) dev_free(sb.hi);
    } else {
      status = gemm_nt_f64(m, n, k, alpha, Ak, ldak, Bk, ldbk, beta, C, st);
    }
  }
  cudaError_t e = cudaStreamSynchronize(st);
  if (tA) dev_free(tA);
  if (tB) dev_free(tB);
  if (status == ACES_OK && e != cudaSuccess) {
    set_error("aces_xgemm: %s", cudaGetErrorString(e));
    status = ACES_ERR_CUDA;
  }
  if (status == ACES_OK && precision == ACES_PREC_BF16X3) {
    if (int tcs = tc_status_and_clear()) {
      set_error("aces_xgemm: tensor-core contraction gave up waiting (code %d)", tcs);
      status = ACES_ERR_TIMEOUT;
    }
  }
  return status;
}

extern "C" int aces_set_wait_limit(double seconds) {
  if (!(seconds > 0.0 && seconds <= 60.0)) {
    set_error("aces_set_wait_limit: %g s outside (0, 60]", seconds);
    return ACES_ERR_ARG;
  }
  return tc_set_wait_limit((unsigned long long)(seconds * 1e9));
}

extern "C" int aces_set_tc_pairs(int on) {
  if (on != 0 && on != 1) {
    set_error("aces_set_tc_pairs: %d (0 or 1)", on);
    return ACES_ERR_ARG;
  }
  tc_set_pairs(on);
  return ACES_OK;
}

extern "C" int aces_set_tc_wide(int on) {
  if (on != 0 && on != 1) {
    set_error("aces_set_tc_wide: %d (0 or 1)", on);
    return ACES_ERR_ARG;
  }
  tc_set_wide(on);
  return ACES_OK;
}

extern "C" int aces_set_autotune(int mode) {
  if (mode < 0 || mode > 2) {
    set_error("aces_set_autotune: mode %d (0, 1 or 2)", mode);
    return ACES_ERR_ARG;
  }
  if (mode == 2) {
    tc_autotune_reset();
    return ACES_OK;
  }
  tc_set_autotune(mode);
  return ACES_OK;
}

extern "C" int aces_autotune_stats(long long *classes, long long *changed, double *tune_ms) {
  tc_autotune_stats(classes, changed, tune_ms);
  return ACES_OK;
}

extern "C" int aces_autotune_save(const char *path) { return tc_autotune_save(path); }

extern "C" int aces_autotune_load(const char *path) { return tc_autotune_load(path); }

extern "C" int aces_debug_inject(int mode) {
  if (mode != 0 && mode != 1) {
    set_error("aces_debug_inject: mode %d (0 or 1)", mode);
    return ACES_ERR_ARG;
  }
  return tc_set_inject(mode);
}
