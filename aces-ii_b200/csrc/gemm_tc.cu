// gemm_tc.cu -- split-precision (BF16x3) operand packing and the tcgen05
// contraction kernel.
#include <cuda_bf16.h>

#include "common.cuh"
#include "gemm.cuh"

namespace acesb200 {

// hi = bf16(x) (round to nearest even), lo = bf16(x - hi); padding is zero.
__global__ void k_split_pack(__nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo,
                             const double *__restrict__ src, long long ld, int rows, int k,
                             int rows_pad, int k_pad) {
  long long total = (long long)rows_pad * k_pad;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    int r = (int)(idx / k_pad), c = (int)(idx % k_pad);
    float x = 0.f;
    double xd = 0.0;
    if (r < rows && c < k) xd = src[(long long)r * ld + c];
    x = (float)xd;
    __nv_bfloat16 h = __float2bfloat16_rn(x);
    float rem = (float)(xd - (double)__bfloat162float(h));
    hi[idx] = h;
    lo[idx] = __float2bfloat16_rn(rem);
  }
}

int split_pack(SplitOperand &op, const double *src, long long ld, int rows, int k,
               cudaStream_t st) {
  int rp = (rows + kSplitRowPad - 1) / kSplitRowPad * kSplitRowPad;
  int kp = (k + kSplitKPad - 1) / kSplitKPad * kSplitKPad;
  size_t need = (size_t)rp * kp * 2 * 2;
  if (!op.hi || op.bytes() < need) {
    if (op.hi) cudaFree(op.hi);
    op.hi = op.lo = nullptr;
    void *p = nullptr;
    if (cudaMalloc(&p, need) != cudaSuccess) {
      cudaGetLastError();
      set_error("split_pack: cudaMalloc %zu failed", need);
      return ACES_ERR_NOMEM;
    }
    op.hi = p;
    op.rows_pad = rp;
    op.k_pad = kp;
  }
  op.rows = rows;
  op.k = k;
  op.rows_pad = rp;
  op.k_pad = kp;
  op.lo = (char *)op.hi + (size_t)rp * kp * 2;
  long long total = (long long)rp * kp;
  long long nb = (total + 255) / 256;
  if (nb > 148 * 32) nb = 148 * 32;
  k_split_pack<<<(unsigned)nb, 256, 0, st>>>((__nv_bfloat16 *)op.hi, (__nv_bfloat16 *)op.lo, src,
                                             ld, rows, k, rp, kp);
  ACES_CUDA(cudaGetLastError());
  return ACES_OK;
}

int gemm_nt_bf16x3(const SplitOperand &A, const SplitOperand &B, int M, int N, double alpha,
                   double beta, const CView &C, cudaStream_t st) {
  (void)A; (void)B; (void)M; (void)N; (void)alpha; (void)beta; (void)C; (void)st;
  set_error("BF16x3 contraction not available in this build");
  return ACES_ERR_UNSUPPORTED;
}

}  // namespace acesb200
