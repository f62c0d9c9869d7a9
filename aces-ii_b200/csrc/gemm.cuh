// gemm.cuh -- contraction kernels of the CC engine.
//
// Every tensor contraction of the CCSD/(T)/Lambda terms is issued as an
// "NT" product over K-contiguous operands (the reference's XGEMM calls,
// tools/xgemm.F:10, after its SSTGEN/SYMTR resorts):
//
//   C[m,n] = alpha * sum_k A[m*lda + k] * B[n*ldb + k] + beta * C[m,n]
//
// with C addressed through a two-level view so a resorted output can be
// written in place:
//   &C[m,n] = p + (m / mdiv)*sm1 + (m % mdiv)*sm0 + (n / ndiv)*sn1 + (n % ndiv)*sn0
#pragma once
#include <cuda_runtime.h>
#ifdef __CUDACC__
#include <cuda_bf16.h>
#endif

namespace acesb200 {

struct CView {
  double *p;
  long long mdiv, sm1, sm0;
  long long ndiv, sn1, sn0;
};

// Offset of index i along one view dimension: (i / div) * s1 + (i % div) * s0.
// Divisors above 2^31 mean a single-level dimension; the others take a 32-bit
// division (a 64-bit one costs several times more per output element).
__host__ __device__ __forceinline__ long long cview_dim(long long div, long long s1,
                                                        long long s0, int i) {
  if (div > 0x7fffffff) return (long long)i * s0;
  const int d = (int)div, q = i / d;
  return (long long)q * s1 + (long long)(i - q * d) * s0;
}
// plain row-major C[m*ldc + n]
inline CView cview_rowmajor(double *p, long long ldc) {
  return CView{p, 1LL << 62, 0, ldc, 1LL << 62, 0, 1};
}
// column-major C[m + n*ldc]
inline CView cview_colmajor(double *p, long long ldc) {
  return CView{p, 1LL << 62, 0, 1, 1LL << 62, 0, ldc};
}
__host__ __device__ __forceinline__ long long cview_off(const CView &C, int m, int n) {
  return cview_dim(C.mdiv, C.sm1, C.sm0, m) + cview_dim(C.ndiv, C.sn1, C.sn0, n);
}

// Walks i = i0, i0+1, ... along one view dimension (divisor div, strides s1,
// s0) without dividing per step (the epilogues' inner loops).
struct ViewWalk {
  long long off, s1, s0;
  int r, d;
  __device__ __forceinline__ ViewWalk(long long div, long long s1_, long long s0_, int i0)
      : s1(s1_), s0(s0_) {
    if (div > 0x7fffffff) {
      d = 0x7fffffff;
      r = 0;
      off = (long long)i0 * s0;
    } else {
      d = (int)div;
      const int q = i0 / d;
      r = i0 - q * d;
      off = (long long)q * s1 + (long long)r * s0;
    }
  }
  __device__ __forceinline__ void next() {
    if (++r == d) {
      r = 0;
      off += s1 - (long long)(d - 1) * s0;
    } else {
      off += s0;
    }
  }
};
struct CViewNWalk : ViewWalk {
  __device__ __forceinline__ CViewNWalk(const CView &C, int n0)
      : ViewWalk(C.ndiv, C.sn1, C.sn0, n0) {}
};

// FP64 tensor-core (DMMA) contraction.
int gemm_nt_f64(int M, int N, int K, double alpha, const double *A, long long lda,
                const double *B, long long ldb, double beta, const CView &C, cudaStream_t st);

// FP64 matrix-vector product y = alpha * A x + beta * y written through C at
// (m, 0) (or (0, m) when transpose_out).
int gemv_f64(int M, int K, double alpha, const double *A, long long lda, const double *x,
             double beta, const CView &C, bool transpose_out, cudaStream_t st);
// gemm_nt_f64 with all scratch (split-K partials) taken from `ws` (capacity
// `cap` doubles); allocates nothing.
int gemm_nt_f64_scratch(int M, int N, int K, double alpha, const double *A, long long lda,
                        const double *B, long long ldb, double beta, const CView &C,
                        double *ws, size_t cap, cudaStream_t st);
// split-K support shared by the contraction kernels
double *splitk_workspace(size_t doubles);
// C = alpha * sum_z part[z] + beta * C; part[z] is [M][N] row-major, or
// [N][M] (m fastest) with mfast
int splitk_reduce(const CView &C, const double *part, int M, int N, int Z, double alpha,
                  double beta, cudaStream_t st, bool mfast = false);

// Split-precision operand: x ~= hi + lo with hi = bf16(x), lo = bf16(x - hi),
// stored K-contiguous with K zero-padded to k_pad.  rows_pad is the row extent
// of the TMA tensor map (= rows): the rows of a 128-row box past it are
// zero-filled by the TMA unit, so thin operands need no padding in memory.
struct SplitOperand {
  void *hi = nullptr;   // __nv_bfloat16[rows_pad * k_pad]
  void *lo = nullptr;
  int rows = 0, k = 0, rows_pad = 0, k_pad = 0;
  size_t cap = 0;       // bytes allocated at hi (both planes)
};

// K padding of split operands (the tcgen05 kernel's k tile)
constexpr int kSplitKPad = 64;

#ifdef __CUDACC__
// the two BF16 planes of one FP64 value: hi = bf16(x) (round to nearest even
// through FP32), lo = bf16(x - hi); every producer of split operands uses it,
// so a fused resort and split_pack give bit-identical planes
__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16 &h, __nv_bfloat16 &l) {
  h = __float2bfloat16_rn((float)x);
  l = __float2bfloat16_rn((float)(x - (double)__bfloat162float(h)));
}
#endif

// Fill a split operand from an FP64 K-contiguous matrix (src[r*ld + k]).
int split_pack(SplitOperand &op, const double *src, long long ld, int rows, int k, cudaStream_t st);

// BF16x3 contraction on tcgen05: A, B split operands with equal k_pad.
// acc = A_hi B_hi + A_hi B_lo + A_lo B_hi in FP32 (TMEM), C = alpha*acc + beta*C (FP64).
int gemm_nt_bf16x3(const SplitOperand &A, const SplitOperand &B, int M, int N, double alpha,
                   double beta, const CView &C, cudaStream_t st);
// Sum of up to 4 split products over one output: C = alpha sum_s A[s] B[s]^T
// + beta C (K segments of a single launch; every A[s] has >= M rows and every
// B[s] >= N rows, each segment its own K)
int gemm_nt_bf16x3_multi(const SplitOperand *A, const SplitOperand *B, int nseg, int M, int N,
                         double alpha, double beta, const CView &C, cudaStream_t st);

// Up to 3 independent products in one persistent launch (no split K):
// C_g = alpha sum_s A_g[s] B_g[s]^T + beta C_g.  The tiles of all problems are
// scheduled together, so products whose own tile counts leave SMs idle in
// their last wave fill each other's.
struct GroupedProblem {
  const SplitOperand *A, *B;  // nseg operands each
  int nseg, M, N;
  CView C;
};
int gemm_nt_bf16x3_grouped(const GroupedProblem *probs, int nprob, double alpha, double beta,
                           cudaStream_t st);

// Batched products over row windows of shared parent operands: entry e
// computes C_e = alpha sum_s A_s[rowA[s] + m, :] B_s[rowB[s] + n, :]^T
// + beta C_e for m < M, n < N, with C_e = the view C shifted by coff
// elements.  All entries share the parents' tensor maps; one launch walks the
// tiles of every entry (the side with fewer tiles fastest, then the entry,
// then the other side, so that entries sharing an operand window read it from
// DRAM once).  With f32out the output is FP32 (beta 0 or 1 only).
constexpr int kBatchSeg = 4;
struct alignas(16) BatchEntry {   // 48 bytes: the kernel reads the rows as two int4
  int rowA[kBatchSeg], rowB[kBatchSeg];
  long long coff;
};
static_assert(sizeof(BatchEntry) == 48, "batch entry layout");
// d_entries: device array of nbatch entries; h_entries: the same on the host
// (checked: every window lies inside its parent)
int gemm_nt_bf16x3_batched(const SplitOperand *Apar, const SplitOperand *Bpar, int nseg, int M,
                           int N, const BatchEntry *h_entries, const BatchEntry *d_entries,
                           int nbatch, double alpha, double beta, const CView &C, bool f32out,
                           cudaStream_t st);

// Rows [row0, row0 + rows) of a split operand (no copy).  The view's tensor
// map ends at the parent's padded rows; rows past the view inside it belong
// to the next slice and only reach output rows that callers discard.
SplitOperand split_view(const SplitOperand &p, int row0, int rows);

// Error code recorded by a tcgen05 kernel whose bounded wait expired (0 = ok);
// reading it clears it.
int tc_status_and_clear();
// Bound (ns) of every mbarrier wait of the tcgen05 kernels on the current
// device, and the test-only fault injection (producer issues no copies).
int tc_set_wait_limit(unsigned long long ns);
int tc_set_inject(int on);
// launches of products with >= 256 rows on CTA pairs (process-wide)
void tc_set_pairs(int on);
// 128 x 256 tiles for the single-chunk FP32-output launches (process-wide)
void tc_set_wide(int on);
// whether a batched FP32-output launch over these K segments with N output
// columns runs on the 128 x 256 tiles (the knob is on, 144 < N <= 256 and
// the segments' k tiles form one chunk)
bool bf16x3_wide_applies(const SplitOperand *A, int nseg, int N);
// tile autotuner of the tensor-core launches (process-wide switch; choices
// cached per device and shape class): on/off, forget every choice, and the
// number of classes tuned, how many of them left the default variant, and the
// device ms their timed runs took
void tc_set_autotune(int on);
void tc_autotune_reset();
void tc_autotune_stats(long long *classes, long long *changed, double *ms);
// the current device's cached choices to / from a text file
int tc_autotune_save(const char *path);
int tc_autotune_load(const char *path);

}  // namespace acesb200
