// xgemm_static.cu -- aces_xgemm_static: the FP64 XGEMM with no device
// allocation, for hosts that cannot call cudaMalloc.
//
// Some callers of this library cannot allocate device memory at the moment
// they want a contraction: a host application that has handed all device
// memory to its own allocator at start-up (a framework's caching allocator,
// or a Fortran driver that reserves one heap up front the way ACES reserves
// its ICORE heap), or a caller in a section where an allocation's implicit
// device synchronisation or possible failure is not acceptable.  This entry
// point therefore draws all of its scratch from one file-scope device array
// of fixed size that every GPU loading the library holds until the process
// exits.
//
// Scratch per call (doubles): m*k for op(A) when transa = 'N' (it is copied
// into the K-contiguous form the kernels read), n*k for op(B) when
// transb = 'T', plus split-K partial sums that are only used when they fit in
// what is left (otherwise the contraction runs unsplit).  Calls needing more
// than kStaticScratchDoubles return ACES_ERR_ARG.  Every call shares the
// array: calls that overlap on the GPU (several host threads, or several
// streams) race on it.  Each call writes every scratch element it reads
// before reading it, so nothing has to start at zero.
#include <algorithm>
#include <cctype>
#include <map>
#include <mutex>

#include "common.cuh"
#include "gemm.cuh"
#include "kernels.cuh"

namespace {

constexpr size_t kStaticScratchDoubles = size_t(1) << 20;  // 8 MiB per device

static __device__ __align__(256) double g_xgemm_scratch[kStaticScratchDoubles];

// Device address of g_xgemm_scratch for the current device, looked up once per
// device with that device current.  (In host code the symbol itself is only
// a host-side stand-in, never a device address.)
int scratch_address(double **out) {
  static std::mutex mu;
  static std::map<int, double *> addr;
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    acesb200::set_error("aces_xgemm_static: cudaGetDevice: %s", cudaGetErrorString(e));
    return ACES_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lk(mu);
  auto it = addr.find(dev);
  if (it != addr.end()) {
    *out = it->second;
    return ACES_OK;
  }
  void *p = nullptr;
  e = cudaGetSymbolAddress(&p, g_xgemm_scratch);
  if (e != cudaSuccess || p == nullptr) {
    acesb200::set_error("aces_xgemm_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    return ACES_ERR_CUDA;
  }
  addr[dev] = static_cast<double *>(p);
  *out = static_cast<double *>(p);
  return ACES_OK;
}

// dst[r*cols + c] = src[r + c*ld] (column-major rows x cols -> K-contiguous)
int to_kmajor_into(double *dst, const double *src, int rows, int cols, long long ld,
                   cudaStream_t st) {
  acesb200::PermSpec s;
  s.n[0] = 1; s.n[1] = 1; s.n[2] = rows; s.n[3] = cols;
  s.nterms = 1;
  s.beta = 0.0;
  s.t[0].src = src;
  s.t[0].alpha = 1.0;
  s.t[0].s[0] = 0; s.t[0].s[1] = 0; s.t[0].s[2] = 1; s.t[0].s[3] = ld;
  return acesb200::permute(dst, s, st);
}

}  // namespace

using namespace acesb200;

extern "C" int aces_xgemm_static(char transa, char transb, int m, int n, int k, double alpha,
                                 const double *A, int lda, const double *B, int ldb, double beta,
                                 double *Cm, int ldc) {
  char ta = (char)toupper(transa), tb = (char)toupper(transb);
  if ((ta != 'N' && ta != 'T') || (tb != 'N' && tb != 'T') || m < 0 || n < 0 || k < 0) {
    set_error("aces_xgemm_static: bad arguments");
    return ACES_ERR_ARG;
  }
  if ((long long)m * n == 0) return ACES_OK;
  if (ldc < (m > 1 ? m : 1)) {
    set_error("aces_xgemm_static: ldc < m");
    return ACES_ERR_ARG;
  }
  // leading dimensions as DGEMM checks them: op(A) is m x k, op(B) is k x n
  if (lda < std::max(1, ta == 'N' ? m : k) || ldb < std::max(1, tb == 'N' ? k : n)) {
    set_error("aces_xgemm_static: lda %d or ldb %d below the operand's row count", lda, ldb);
    return ACES_ERR_ARG;
  }
  size_t need = (ta == 'N' ? (size_t)m * k : 0) + (tb == 'T' ? (size_t)n * k : 0);
  if (need > kStaticScratchDoubles) {
    set_error("aces_xgemm_static: operands need %zu scratch doubles, the static limit is %zu "
              "(use aces_xgemm)", need, kStaticScratchDoubles);
    return ACES_ERR_ARG;
  }
  double *scratch = nullptr;
  ACES_TRY(scratch_address(&scratch));
  cudaStream_t st = 0;
  const double *Ak = A, *Bk = B;
  long long ldak = lda, ldbk = ldb;
  size_t used = 0;
  if (ta == 'N') {
    ACES_TRY(to_kmajor_into(scratch, A, m, k, lda, st));
    Ak = scratch;
    ldak = k;
    used += (size_t)m * k;
  }
  if (tb == 'T') {
    ACES_TRY(to_kmajor_into(scratch + used, B, n, k, ldb, st));
    Bk = scratch + used;
    ldbk = k;
    used += (size_t)n * k;
  }
  // split-K partials start on a 256-byte boundary after the operand copies
  used = (used + 31) / 32 * 32;
  double *ws = scratch + used;
  size_t cap = used < kStaticScratchDoubles ? kStaticScratchDoubles - used : 0;
  int status = gemm_nt_f64_scratch(m, n, k, alpha, Ak, ldak, Bk, ldbk, beta,
                                   cview_colmajor(Cm, ldc), ws, cap, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (status == ACES_OK && e != cudaSuccess) {
    set_error("aces_xgemm_static: %s", cudaGetErrorString(e));
    status = ACES_ERR_CUDA;
  }
  return status;
}
