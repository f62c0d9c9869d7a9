// gemm_f64.cu -- FP64 contraction on the DMMA tensor-core path
// (mma.sync.m8n8k4.f64): the plain-FP64 comparator of the engine and the
// arithmetic of the reference's XGEMM -> DGEMM (tools/xgemm.F:10-49).
//
// Tile 128 x 128 x 16, 256 threads (8 warps as 2 x 4, each warp 64 x 32), a
// 4-stage cp.async pipeline (three k tiles in flight while one is computed,
// one barrier per k tile), padded shared-memory rows (20 doubles) so the
// fragment loads of a half-warp hit 32 distinct banks.
#include <algorithm>

#include "common.cuh"
#include "gemm.cuh"

namespace acesb200 {

namespace {
constexpr int BM = 128, BN = 128, BK = 16, LDS = BK + 4;
constexpr int kThreads = 256;
constexpr int kStages = 4;
constexpr int kStageDoubles = (BM + BN) * LDS;
constexpr int kSmemBytes = kStages * kStageDoubles * 8;
static_assert(kSmemBytes <= 227 * 1024, "pipeline depth");

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

template <int VEC>
__device__ __forceinline__ void cp_async(double *dst, const double *src, bool valid) {
  unsigned d = smem_u32(dst);
  int sz = valid ? VEC * 8 : 0;
  if (VEC == 2)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(sz));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(sz));
}

__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// The copies of one operand tile (BM rows x BK doubles) in VEC-double chunks:
// thread t always takes the chunks of k offset kc = (t % CPR) * VEC in rows
// t / CPR + i * RS, so the row pointers, their bounds and the shared-memory
// offsets are computed once per block; a k tile then adds its k0 and tests
// one K bound.
template <int VEC>
struct CopyPlan {
  static constexpr int CPR = BK / VEC;          // chunks per row
  static constexpr int RS = kThreads / CPR;     // row step between a thread's chunks
  static constexpr int kPer = BM / RS;          // chunks per thread and operand
  const double *row[kPer];                      // &X[row][kc] (X itself for rows past the end)
  unsigned live;                                // bit i: row i inside the operand
  int kc, soff0;                                // k offset; shared offset of chunk 0
  __device__ __forceinline__ CopyPlan(const double *X, long long ld, int rows, int r0base) {
    const int t = threadIdx.x;
    kc = (t % CPR) * VEC;
    const int r0 = t / CPR;
    soff0 = r0 * LDS + kc;
    live = 0;
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int gr = r0base + r0 + i * RS;
      const bool ok = gr < rows;
      row[i] = ok ? X + (long long)gr * ld + kc : X;
      live |= ok ? 1u << i : 0u;
    }
  }
  __device__ __forceinline__ void issue(double *stage, const double *X, int k0, int ke) const {
    const bool kok = k0 + kc < ke;
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const bool v = kok && ((live >> i) & 1u);
      cp_async<VEC>(stage + soff0 + i * RS * LDS, v ? row[i] + k0 : X, v);
    }
  }
};
static_assert(BM == BN, "one copy plan shape for both operands");

template <int VEC>
__global__ void __launch_bounds__(kThreads, 1)
    k_gemm_nt_f64(int M, int N, int K, double alpha, const double *__restrict__ A, long long lda,
                  const double *__restrict__ B, long long ldb, double beta, CView C, int kchunk,
                  double *__restrict__ part) {
  extern __shared__ double smem[];
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warps
  const int lr = lane >> 2, lc = lane & 3;
  double acc[8][4][2];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  // split-K: blockIdx.z owns K range [kb, ke)
  const int kb = blockIdx.z * kchunk;
  const int ke = min(K, kb + kchunk);
  const int nk = ke > kb ? (ke - kb + BK - 1) / BK : 0;
  auto stA = [&](int s) { return smem + s * kStageDoubles; };
  auto stB = [&](int s) { return smem + s * kStageDoubles + BM * LDS; };
  const CopyPlan<VEC> pa(A, lda, M, m0), pb(B, ldb, N, n0);
  // prologue: k tiles 0 .. kStages-2 in flight (one commit group each, empty
  // groups past the end keep the count uniform)
#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nk) {
      pa.issue(stA(s), A, kb + s * BK, ke);
      pb.issue(stB(s), B, kb + s * BK, ke);
    }
    cp_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    // group kt complete: at most kStages-2 younger groups still pending
    cp_wait<kStages - 2>();
    __syncthreads();
    // refill the slot computed in the previous iteration (every thread is past it)
    const int nxt = kt + kStages - 1;
    if (nxt < nk) {
      pa.issue(stA(nxt % kStages), A, kb + nxt * BK, ke);
      pb.issue(stB(nxt % kStages), B, kb + nxt * BK, ke);
    }
    cp_commit();
    const double *a_s = stA(kt % kStages) + (wm * 64) * LDS;
    const double *b_s = stB(kt % kStages) + (wn * 32) * LDS;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double af[8], bf[4];
#pragma unroll
      for (int i = 0; i < 8; ++i) af[i] = a_s[(i * 8 + lr) * LDS + kk + lc];
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = b_s[(j * 8 + lr) * LDS + kk + lc];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
  }
  cp_wait0();
  if (part) {
    // split-K partial: dense [z][M][N]
    double *pz = part + (size_t)blockIdx.z * M * N;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      int m = m0 + wm * 64 + i * 8 + lr;
      if (m >= M) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          int n = n0 + wn * 32 + j * 8 + lc * 2 + h;
          if (n < N) pz[(size_t)m * N + n] = acc[i][j][h];
        }
    }
    return;
  }
  // epilogue through the two-level output view; the beta*C loads of a row
  // are issued together before its stores
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    int m = m0 + wm * 64 + i * 8 + lr;
    if (m >= M) continue;
    long long mo = cview_dim(C.mdiv, C.sm1, C.sm0, m);
    double old[4][2];
    if (beta != 0.0) {
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          int n = n0 + wn * 32 + j * 8 + lc * 2 + h;
          old[j][h] = n < N ? __ldg(C.p + mo + cview_dim(C.ndiv, C.sn1, C.sn0, n)) : 0.0;
        }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        int n = n0 + wn * 32 + j * 8 + lc * 2 + h;
        if (n >= N) continue;
        double r = alpha * acc[i][j][h];
        if (beta != 0.0) r += beta * old[j][h];
        C.p[mo + cview_dim(C.ndiv, C.sn1, C.sn0, n)] = r;
      }
    }
  }
}
}  // namespace

// C = alpha * sum_z part[z] + beta * C
// part[z][m][n] (mfast false) or part[z][n][m] (mfast true); the slices are
// summed in order z = 0, 1, ... with four of them loaded at a time.  Wide =
// false: M * N below 2^31, the index split with FastDiv (fd: M if mfast, else N).
template <bool Wide>
__global__ void k_splitk_reduce(CView C, const double *__restrict__ part, int M, int N, int Z,
                                double alpha, double beta, bool mfast, FastDiv fd) {
  const long long total = (long long)M * N;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    int m, n;
    if (Wide) {
      m = mfast ? (int)(idx % M) : (int)(idx / N);
      n = mfast ? (int)(idx / M) : (int)(idx % N);
    } else {
      const unsigned q = fd.div((unsigned)idx), r = (unsigned)idx - q * fd.d;
      m = mfast ? (int)r : (int)q;
      n = mfast ? (int)q : (int)r;
    }
    const double *pz = part + idx;
    double s = 0.0;
    int z = 0;
    for (; z + 4 <= Z; z += 4) {
      const double a0 = __ldg(pz), a1 = __ldg(pz + total), a2 = __ldg(pz + 2 * total),
                   a3 = __ldg(pz + 3 * total);
      s += a0;
      s += a1;
      s += a2;
      s += a3;
      pz += 4 * total;
    }
    for (; z < Z; ++z, pz += total) s += __ldg(pz);
    double *cp = C.p + cview_off(C, m, n);
    double r = alpha * s;
    if (beta != 0.0) r += beta * *cp;
    *cp = r;
  }
}

// y[m] = alpha * sum_k A[m*lda + k] x[k] + beta * y[m]; one warp per row
__global__ void k_gemv_f64(int M, int K, double alpha, const double *__restrict__ A,
                           long long lda, const double *__restrict__ x, double beta, CView C,
                           bool transpose_out) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int m = warp; m < M; m += nwarps) {
    const double *a = A + (long long)m * lda;
    // four independent partial sums keep four row loads in flight per lane
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int k = lane;
    for (; k + 96 < K; k += 128) {
      s0 += a[k] * __ldg(x + k);
      s1 += a[k + 32] * __ldg(x + k + 32);
      s2 += a[k + 64] * __ldg(x + k + 64);
      s3 += a[k + 96] * __ldg(x + k + 96);
    }
    for (; k < K; k += 32) s0 += a[k] * __ldg(x + k);
    double s = (s0 + s1) + (s2 + s3);
    for (int off = 16; off; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (lane == 0) {
      int mm = transpose_out ? 0 : m, nn = transpose_out ? m : 0;
      double *cp = C.p + cview_off(C, mm, nn);
      double r = alpha * s;
      if (beta != 0.0) r += beta * *cp;
      *cp = r;
    }
  }
}

// Partial row sums for products with few rows: warp w takes row w / W and
// the w % W-th K chunk of it (kc elements, a multiple of 128); the partials
// go to part[row * W + chunk].
__global__ void k_gemv_part(int M, int K, int W, int kc, const double *__restrict__ A,
                            long long lda, const double *__restrict__ x,
                            double *__restrict__ part) {
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= (long long)M * W) return;  // warp-uniform
  const int m = (int)(warp / W), c = (int)(warp - (long long)m * W);
  const int k0 = c * kc, k1 = min(K, k0 + kc);
  const double *a = A + (long long)m * lda;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int k = k0 + lane;
  for (; k + 96 < k1; k += 128) {
    s0 += a[k] * __ldg(x + k);
    s1 += a[k + 32] * __ldg(x + k + 32);
    s2 += a[k + 64] * __ldg(x + k + 64);
    s3 += a[k + 96] * __ldg(x + k + 96);
  }
  for (; k < k1; k += 32) s0 += a[k] * __ldg(x + k);
  double t = (s0 + s1) + (s2 + s3);
  for (int off = 16; off; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
  if (lane == 0) part[warp] = t;
}

// y[m] = alpha * sum_c part[m * W + c] + beta * y[m], the chunks summed in order
__global__ void k_gemv_final(int M, int W, double alpha, const double *__restrict__ part,
                             double beta, CView C, bool transpose_out) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  double t = 0.0;
  for (int c = 0; c < W; ++c) t += part[(long long)m * W + c];
  const int mm = transpose_out ? 0 : m, nn = transpose_out ? m : 0;
  double *cp = C.p + cview_off(C, mm, nn);
  double r = alpha * t;
  if (beta != 0.0) r += beta * *cp;
  *cp = r;
}

// Tiny products (at most kTinyOut outputs): one warp per output, its lanes
// striding K (coalesced row reads, four independent partial sums per lane),
// reduced by shuffles in a fixed order.
constexpr long long kTinyOut = 8192;
__global__ void k_gemm_tiny_f64(int M, int N, int K, double alpha, const double *__restrict__ A,
                                long long lda, const double *__restrict__ B, long long ldb,
                                double beta, CView C) {
  const int w = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= M * N) return;  // warp-uniform
  const int m = w % M, n = w / M;
  const double *a = A + (long long)m * lda, *b = B + (long long)n * ldb;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int k = lane;
  for (; k + 96 < K; k += 128) {
    s0 += __ldg(a + k) * __ldg(b + k);
    s1 += __ldg(a + k + 32) * __ldg(b + k + 32);
    s2 += __ldg(a + k + 64) * __ldg(b + k + 64);
    s3 += __ldg(a + k + 96) * __ldg(b + k + 96);
  }
  for (; k < K; k += 32) s0 += __ldg(a + k) * __ldg(b + k);
  double t = (s0 + s1) + (s2 + s3);
  for (int off = 16; off; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
  if (lane == 0) {
    double *cp = C.p + cview_off(C, m, n);
    double r = alpha * t;
    if (beta != 0.0) r += beta * *cp;
    *cp = r;
  }
}

// ---------------------------------------------------------------------------
// Thin contractions (one output dimension S <= 32): out(l, s) = sum_k X[l,k] Y[s,k]
// with X the long operand (L rows) and Y the short one.  64 x 32 output tile
// per block, K staged in 32-wide shared-memory chunks, 8 outputs per thread in
// FP64 FMA; split-K over blockIdx.z.  Written to C(m,n) = out(l,s) or out(s,l).
// These products stream their long operand once: bandwidth bound.
// ---------------------------------------------------------------------------
constexpr int TL = 64, TS = 32, TK = 32;

__global__ void __launch_bounds__(256)
    k_gemm_thin_f64(int L, int S, int K, double alpha, const double *__restrict__ X,
                    long long ldx, const double *__restrict__ Y, long long ldy, double beta,
                    CView C, bool s_is_m, int kchunk, double *__restrict__ part) {
  __shared__ double Xs[TL][TK + 1];
  __shared__ double Ys[TS][TK + 1];
  const int l0 = blockIdx.x * TL;
  const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
  const int t = threadIdx.x, r = t >> 3, c = t & 7;
  double acc[2][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  for (int k0 = kb; k0 < ke; k0 += TK) {
    for (int e = t; e < TL * TK; e += 256) {
      int rr = e / TK, kk = e % TK;
      int l = l0 + rr, k = k0 + kk;
      Xs[rr][kk] = (l < L && k < ke) ? X[(long long)l * ldx + k] : 0.0;
    }
    for (int e = t; e < TS * TK; e += 256) {
      int rr = e / TK, kk = e % TK;
      int k = k0 + kk;
      Ys[rr][kk] = (rr < S && k < ke) ? Y[(long long)rr * ldy + k] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < TK; ++kk) {
      double x0 = Xs[2 * r][kk], x1 = Xs[2 * r + 1][kk];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        double y = Ys[4 * c + j][kk];
        acc[0][j] = fma(x0, y, acc[0][j]);
        acc[1][j] = fma(x1, y, acc[1][j]);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    int l = l0 + 2 * r + i;
    if (l >= L) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int sidx = 4 * c + j;
      if (sidx >= S) continue;
      int m = s_is_m ? sidx : l, n = s_is_m ? l : sidx;
      if (part) {
        part[(size_t)blockIdx.z * (size_t)L * S + (size_t)l * S + sidx] = acc[i][j];
        continue;
      }
      double *cp = C.p + cview_off(C, m, n);
      double v = alpha * acc[i][j];
      if (beta != 0.0) v += beta * *cp;
      *cp = v;
    }
  }
}

// Split-K reduction with many slices and few outputs: one warp per output,
// lane k adds slices k, k+32, ..., then a fixed shuffle tree (deterministic).
// layout 0: part[z][m][n]; 1: part[z][n][m]; 2 / 3: part[z][l][s] of the thin
// kernel with (m, n) = (l, s) / (s, l) and S the short dimension.
__global__ void k_reduce_warp(CView C, const double *__restrict__ part, int M, int N, int Z,
                              double alpha, double beta, int layout, int S) {
  const long long total = (long long)M * N;
  const int lane = threadIdx.x & 31;
  for (long long idx = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; idx < total;
       idx += ((long long)gridDim.x * blockDim.x) >> 5) {
    double sum = 0.0;
    for (int z = lane; z < Z; z += 32) sum += part[(size_t)z * total + idx];
    for (int off = 16; off; off >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, off);
    if (lane == 0) {
      int m, n;
      if (layout == 0) {
        m = (int)(idx / N);
        n = (int)(idx % N);
      } else if (layout == 1) {
        m = (int)(idx % M);
        n = (int)(idx / M);
      } else {  // thin partials: idx = l * S + s
        const int l = (int)(idx / S), sidx = (int)(idx % S);
        m = layout == 3 ? sidx : l;
        n = layout == 3 ? l : sidx;
      }
      double *cp = C.p + cview_off(C, m, n);
      double v = alpha * sum;
      if (beta != 0.0) v += beta * *cp;
      *cp = v;
    }
  }
}

static void launch_reduce_warp(const CView &C, const double *part, int M, int N, int Z,
                               double alpha, double beta, int layout, int S, cudaStream_t st) {
  const long long total = (long long)M * N;
  long long nb = (total + 7) / 8;  // 8 warps per block
  if (nb > 148 * 32) nb = 148 * 32;
  k_reduce_warp<<<(unsigned)nb, 256, 0, st>>>(C, part, M, N, Z, alpha, beta, layout, S);
  count_launch();
}

// reduce thin split-K partials part[z][l][s] into C
__global__ void k_thin_reduce(CView C, const double *__restrict__ part, int L, int S, int Z,
                              double alpha, double beta, bool s_is_m) {
  long long total = (long long)L * S;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    int l = (int)(idx / S), sidx = (int)(idx % S);
    double sum = 0.0;
    for (int z = 0; z < Z; ++z) sum += part[(size_t)z * total + idx];
    int m = s_is_m ? sidx : l, n = s_is_m ? l : sidx;
    double *cp = C.p + cview_off(C, m, n);
    double v = alpha * sum;
    if (beta != 0.0) v += beta * *cp;
    *cp = v;
  }
}

// ---------------------------------------------------------------------------
// Low-rank updates (K <= 32): C(m,n) = alpha sum_k A[m,k] B[n,k] + beta C(m,n).
// Output bound.  A block owns 128 outputs along the "fast" index (the one with
// unit stride in the view, so the update of C coalesces) x 32 along the other.
// Both short operands are staged in shared memory with an odd row stride; each
// thread runs 8 independent FMA chains (one per slow index) over k, then
// updates its 8 outputs: one RED per element for beta = 1 on a coalesced view
// (a single owner per element, so the sum equals load + add + store), else a
// batched read-modify-write.
// ---------------------------------------------------------------------------
constexpr int LR_F = 128, LR_S = 32, LR_K = 32;

__global__ void __launch_bounds__(LR_F)
    k_gemm_lowrank_f64(int M, int N, int K, double alpha, const double *__restrict__ A,
                       long long lda, const double *__restrict__ B, long long ldb, double beta,
                       CView C, bool fast_is_m, int tiles_f) {
  extern __shared__ double lr_smem[];
  const int ks = K | 1;  // odd row stride: column reads across threads are conflict free
  double *Fs = lr_smem;              // [LR_F][ks]
  double *Ss = lr_smem + LR_F * ks;  // [LR_S][ks]
  const int nf = fast_is_m ? M : N, ns = fast_is_m ? N : M;
  const double *Fp = fast_is_m ? A : B;
  const double *Sp = fast_is_m ? B : A;
  const long long ldf = fast_is_m ? lda : ldb, lds = fast_is_m ? ldb : lda;
  const int f0 = (blockIdx.x % tiles_f) * LR_F;
  const int s0 = (blockIdx.x / tiles_f) * LR_S;
  for (int e = threadIdx.x; e < LR_F * K; e += LR_F) {
    const int rr = e / K, kk = e - rr * K;
    Fs[rr * ks + kk] = f0 + rr < nf ? Fp[(long long)(f0 + rr) * ldf + kk] : 0.0;
  }
  for (int e = threadIdx.x; e < LR_S * K; e += LR_F) {
    const int rr = e / K, kk = e - rr * K;
    Ss[rr * ks + kk] = s0 + rr < ns ? Sp[(long long)(s0 + rr) * lds + kk] : 0.0;
  }
  __syncthreads();
  const int f = f0 + threadIdx.x;
  if (f >= nf) return;
  const int nsl = min(LR_S, ns - s0);
  // fast and slow view dimensions
  const long long fdiv = fast_is_m ? C.mdiv : C.ndiv, fs1 = fast_is_m ? C.sm1 : C.sn1,
                  fs0 = fast_is_m ? C.sm0 : C.sn0;
  const long long sdiv = fast_is_m ? C.ndiv : C.mdiv, ss1 = fast_is_m ? C.sn1 : C.sm1,
                  ss0 = fast_is_m ? C.sn0 : C.sm0;
  double *const cf = C.p + cview_dim(fdiv, fs1, fs0, f);
  ViewWalk w(sdiv, ss1, ss0, s0);
#ifndef ACES_LR_RED
#define ACES_LR_RED 1
#endif
  const bool red = ACES_LR_RED && beta == 1.0 && fs0 == 1;
  const double *fr = Fs + threadIdx.x * ks;
#pragma unroll 1
  for (int sb = 0; sb < nsl; sb += 8) {
    double acc[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j] = 0.0;
    const double *sr = Ss + sb * ks;  // rows sb..sb+7 < LR_S (zero past ns)
#pragma unroll 4
    for (int k = 0; k < K; ++k) {
      const double fv = fr[k];
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[j] = fma(fv, sr[j * ks + k], acc[j]);
    }
    long long off[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      acc[j] *= alpha;
      off[j] = w.off;
      w.next();
    }
    if (beta == 0.0) {
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (sb + j < nsl) cf[off[j]] = acc[j];
    } else if (red) {
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (sb + j < nsl) atomicAdd(cf + off[j], acc[j]);
    } else {
      double old[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) old[j] = sb + j < nsl ? __ldg(cf + off[j]) : 0.0;
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (sb + j < nsl) cf[off[j]] = acc[j] + beta * old[j];
    }
  }
}

static int launch_lowrank(int M, int N, int K, double alpha, const double *A, long long lda,
                          const double *B, long long ldb, double beta, const CView &C,
                          cudaStream_t st) {
  // run threads along the unit-stride output index
  const bool fast_is_m = C.sm0 == 1 || C.sn0 != 1;
  const int nf = fast_is_m ? M : N, ns = fast_is_m ? N : M;
  const int tiles_f = (nf + LR_F - 1) / LR_F;
  const long long nb = (long long)tiles_f * ((ns + LR_S - 1) / LR_S);
  if (nb > 0x7fffffffLL) {
    set_error("low-rank contraction grid too large (%lld blocks)", nb);
    return ACES_ERR_ARG;
  }
  const size_t smem = (size_t)(LR_F + LR_S) * (K | 1) * sizeof(double);
  k_gemm_lowrank_f64<<<(unsigned)nb, LR_F, smem, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C,
                                                       fast_is_m, tiles_f);
  count_launch();
  ACES_CUDA(cudaGetLastError());
  return ACES_OK;
}

// split-K partials of the current device (one buffer per device, grown on demand)
double *splitk_workspace(size_t doubles) {
  static double *ws[64] = {nullptr};
  static size_t cap[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return nullptr;
  }
  if (doubles > cap[dev]) {
    if (ws[dev]) dev_free(ws[dev]);
    ws[dev] = nullptr;
    cap[dev] = 0;
    if (dev_alloc((void **)&ws[dev], doubles * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    cap[dev] = doubles;
  }
  return ws[dev];
}

int splitk_reduce(const CView &C, const double *part, int M, int N, int Z, double alpha,
                  double beta, cudaStream_t st, bool mfast) {
  long long total = (long long)M * N;
  if (Z >= 24 && total <= 16384) {
    // few outputs, many slices: a warp per output instead of a serial loop
    launch_reduce_warp(C, part, M, N, Z, alpha, beta, mfast ? 1 : 0, 0, st);
    ACES_CUDA(cudaGetLastError());
    return ACES_OK;
  }
  long long nb = (total + 255) / 256;
  if (nb > 148 * 16) nb = 148 * 16;
  const FastDiv fd((unsigned)std::max(1, mfast ? M : N));
  if (total < (1LL << 31))
    k_splitk_reduce<false><<<(unsigned)nb, 256, 0, st>>>(C, part, M, N, Z, alpha, beta, mfast, fd);
  else
    k_splitk_reduce<true><<<(unsigned)nb, 256, 0, st>>>(C, part, M, N, Z, alpha, beta, mfast, fd);
  count_launch();
  ACES_CUDA(cudaGetLastError());
  return ACES_OK;
}

int gemv_f64(int M, int K, double alpha, const double *A, long long lda, const double *x,
             double beta, const CView &C, bool transpose_out, cudaStream_t st) {
  if (M <= 0) return ACES_OK;
  // few rows: each row split over W warps (about 4736 warps in all, K chunks
  // of at least 128), so the matrix streams with enough loads in flight
  const long long kTargetWarps = 148 * 32;
  if (M <= kTargetWarps && K >= 256) {
    int W = (int)std::min<long long>(32, (kTargetWarps + M - 1) / M);
    int kc = ((K + W - 1) / W + 127) / 128 * 128;
    W = (K + kc - 1) / kc;
    if (W > 1) {
      double *part = splitk_workspace((size_t)M * W);
      if (!part) {
        set_error("gemv: partial-sum workspace allocation failed");
        return ACES_ERR_NOMEM;
      }
      const long long nw = (long long)M * W;
      k_gemv_part<<<(unsigned)((nw * 32 + 255) / 256), 256, 0, st>>>(M, K, W, kc, A, lda, x,
                                                                      part);
      count_launch();
      k_gemv_final<<<(unsigned)((M + 255) / 256), 256, 0, st>>>(M, W, alpha, part, beta, C,
                                                                transpose_out);
      count_launch();
      ACES_CUDA(cudaGetLastError());
      return ACES_OK;
    }
  }
  long long warps = M;
  long long nb = (warps * 32 + 255) / 256;
  if (nb > 148 * 32) nb = 148 * 32;
  k_gemv_f64<<<(unsigned)nb, 256, 0, st>>>(M, K, alpha, A, lda, x, beta, C, transpose_out);
  count_launch();
  ACES_CUDA(cudaGetLastError());
  return ACES_OK;
}

int gemm_nt_f64(int M, int N, int K, double alpha, const double *A, long long lda,
                const double *B, long long ldb, double beta, const CView &C, cudaStream_t st) {
  if (M <= 0 || N <= 0) return ACES_OK;
  if (K <= 0) {
    // C = beta*C: run with K = 0 is a scale; issue through the kernel with no k tiles
  }
  // a few thousand outputs: one warp each (no tiles, no split K)
  if ((long long)M * N <= kTinyOut && K > 0 && K <= 8192) {
    k_gemm_tiny_f64<<<(unsigned)(((long long)M * N * 32 + 255) / 256), 256, 0, st>>>(
        M, N, K, alpha, A, lda, B, ldb, beta, C);
    count_launch();
    ACES_CUDA(cudaGetLastError());
    return ACES_OK;
  }
  // K <= 32: output-bound low-rank update
  if (K <= LR_K) return launch_lowrank(M, N, K, alpha, A, lda, B, ldb, beta, C, st);
  // one output dimension <= 32: thin kernel over the long dimension
  if (M <= TS || N <= TS) {
    bool s_is_m = M <= TS && (M <= N);
    int L = s_is_m ? N : M, S = s_is_m ? M : N;
    const double *X = s_is_m ? B : A;
    const double *Y = s_is_m ? A : B;
    long long ldx = s_is_m ? ldb : lda, ldy = s_is_m ? lda : ldb;
    long long lt = (L + TL - 1) / TL;
    int Z = 1, kchunk = K;
    double *part = nullptr;
    if (lt < 592 && K >= 4 * TK) {
      Z = (int)std::min<long long>((592 + lt - 1) / lt, K / (2 * TK));
      if (Z > 1) {
        kchunk = ((K + Z - 1) / Z + TK - 1) / TK * TK;
        Z = (K + kchunk - 1) / kchunk;
        part = splitk_workspace((size_t)Z * L * S);
        if (!part) {
          set_error("gemm thin: split-K workspace allocation failed");
          return ACES_ERR_NOMEM;
        }
      }
    }
    dim3 g((unsigned)lt, 1, Z);
    k_gemm_thin_f64<<<g, 256, 0, st>>>(L, S, K, alpha, X, ldx, Y, ldy, beta, C, s_is_m, kchunk,
                                       Z > 1 ? part : nullptr);
    count_launch();
    ACES_CUDA(cudaGetLastError());
    if (Z >= 24 && (long long)L * S <= 16384) {
      launch_reduce_warp(C, part, M, N, Z, alpha, beta, s_is_m ? 3 : 2, S, st);
      ACES_CUDA(cudaGetLastError());
    } else if (Z > 1) {
      long long total = (long long)L * S;
      long long nb = (total + 255) / 256;
      if (nb > 148 * 16) nb = 148 * 16;
      k_thin_reduce<<<(unsigned)nb, 256, 0, st>>>(C, part, L, S, Z, alpha, beta, s_is_m);
      count_launch();
      ACES_CUDA(cudaGetLastError());
    }
    return ACES_OK;
  }
  static bool attr_set[64] = {false};  // the shared-memory opt-in is per device
  int dev = 0;
  ACES_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("gemm_nt_f64: device %d outside 0..63", dev);
    return ACES_ERR_ARG;
  }
  if (!attr_set[dev]) {
    ACES_CUDA(cudaFuncSetAttribute(k_gemm_nt_f64<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   kSmemBytes));
    ACES_CUDA(cudaFuncSetAttribute(k_gemm_nt_f64<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   kSmemBytes));
    attr_set[dev] = true;
  }
  dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
  if (grid.y > 65535) {
    set_error("gemm_nt_f64: M=%d too large", M);
    return ACES_ERR_ARG;
  }
  // split K when the output has too few tiles to fill the GPU
  int Z = 1;
  long long tiles = (long long)grid.x * grid.y;
  int nkt = (K + BK - 1) / BK;
  if (tiles < 148 && nkt >= 16) {
    Z = (int)std::min<long long>((296 + tiles - 1) / tiles, nkt / 8);
    if (Z < 1) Z = 1;
  }
  int kchunk = K;
  double *part = nullptr;
  if (Z > 1) {
    kchunk = ((K + Z - 1) / Z + BK - 1) / BK * BK;
    Z = (K + kchunk - 1) / kchunk;
    part = splitk_workspace((size_t)Z * M * N);
    if (!part) {
      set_error("gemm_nt_f64: split-K workspace allocation failed");
      return ACES_ERR_NOMEM;
    }
    grid.z = Z;
  }
  bool vec2 = (lda % 2 == 0) && (ldb % 2 == 0) && (K % 2 == 0) &&
              ((reinterpret_cast<uintptr_t>(A) & 15) == 0) &&
              ((reinterpret_cast<uintptr_t>(B) & 15) == 0);
  if (kchunk % 2) vec2 = false;
  if (vec2)
    k_gemm_nt_f64<2><<<grid, kThreads, kSmemBytes, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C,
                                                         kchunk, part);
  else
    k_gemm_nt_f64<1><<<grid, kThreads, kSmemBytes, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C,
                                                         kchunk, part);
  count_launch();
  ACES_CUDA(cudaGetLastError());
  if (part) return splitk_reduce(C, part, M, N, Z, alpha, beta, st);
  return ACES_OK;
}

}  // namespace acesb200

namespace acesb200 {

// The same FP64 contraction dispatch as gemm_nt_f64, with every scratch
// buffer taken from caller-provided device memory `ws` (capacity `cap`
// doubles) instead of the library's allocated workspace.  Split-K is reduced
// to what fits; when even the unsplit form needs no scratch it runs unsplit.
int gemm_nt_f64_scratch(int M, int N, int K, double alpha, const double *A, long long lda,
                        const double *B, long long ldb, double beta, const CView &C,
                        double *ws, size_t cap, cudaStream_t st) {
  if (M <= 0 || N <= 0) return ACES_OK;
  if (K <= LR_K) return launch_lowrank(M, N, K, alpha, A, lda, B, ldb, beta, C, st);
  if (M <= TS || N <= TS) {
    bool s_is_m = M <= TS && (M <= N);
    int L = s_is_m ? N : M, S = s_is_m ? M : N;
    const double *X = s_is_m ? B : A;
    const double *Y = s_is_m ? A : B;
    long long ldx = s_is_m ? ldb : lda, ldy = s_is_m ? lda : ldb;
    long long lt = (L + TL - 1) / TL;
    int Z = 1, kchunk = K;
    if (lt < 592 && K >= 4 * TK) {
      long long zfit = (long long)(cap / ((size_t)L * S));
      Z = (int)std::min<long long>(std::min<long long>((592 + lt - 1) / lt, K / (2 * TK)), zfit);
      if (Z > 1) {
        kchunk = ((K + Z - 1) / Z + TK - 1) / TK * TK;
        Z = (K + kchunk - 1) / kchunk;
      } else {
        Z = 1;
        kchunk = K;
      }
    }
    dim3 g((unsigned)lt, 1, Z);
    k_gemm_thin_f64<<<g, 256, 0, st>>>(L, S, K, alpha, X, ldx, Y, ldy, beta, C, s_is_m, kchunk,
                                       Z > 1 ? ws : nullptr);
    count_launch();
    ACES_CUDA(cudaGetLastError());
    if (Z > 1) {
      long long total = (long long)L * S;
      long long nb = (total + 255) / 256;
      if (nb > 148 * 16) nb = 148 * 16;
      k_thin_reduce<<<(unsigned)nb, 256, 0, st>>>(C, ws, L, S, Z, alpha, beta, s_is_m);
      count_launch();
      ACES_CUDA(cudaGetLastError());
    }
    return ACES_OK;
  }
  ACES_CUDA(cudaFuncSetAttribute(k_gemm_nt_f64<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kSmemBytes));
  ACES_CUDA(cudaFuncSetAttribute(k_gemm_nt_f64<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kSmemBytes));
  dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
  if (grid.y > 65535) {
    set_error("gemm_nt_f64_scratch: M=%d too large", M);
    return ACES_ERR_ARG;
  }
  int Z = 1;
  long long tiles = (long long)grid.x * grid.y;
  int nkt = (K + BK - 1) / BK;
  if (tiles < 148 && nkt >= 16) {
    long long zfit = (long long)(cap / ((size_t)M * N));
    Z = (int)std::min<long long>(std::min<long long>((296 + tiles - 1) / tiles, nkt / 8), zfit);
    if (Z < 1) Z = 1;
  }
  int kchunk = K;
  double *part = nullptr;
  if (Z > 1) {
    kchunk = ((K + Z - 1) / Z + BK - 1) / BK * BK;
    Z = (K + kchunk - 1) / kchunk;
    part = ws;
    grid.z = Z;
  }
  bool vec2 = (lda % 2 == 0) && (ldb % 2 == 0) && (K % 2 == 0) &&
              ((reinterpret_cast<uintptr_t>(A) & 15) == 0) &&
              ((reinterpret_cast<uintptr_t>(B) & 15) == 0);
  if (kchunk % 2) vec2 = false;
  if (vec2)
    k_gemm_nt_f64<2><<<grid, kThreads, kSmemBytes, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C,
                                                         kchunk, part);
  else
    k_gemm_nt_f64<1><<<grid, kThreads, kSmemBytes, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C,
                                                         kchunk, part);
  count_launch();
  ACES_CUDA(cudaGetLastError());
  if (part) return splitk_reduce(C, part, M, N, Z, alpha, beta, st);
  return ACES_OK;
}

}  // namespace acesb200
