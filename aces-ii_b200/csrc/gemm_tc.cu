// gemm_tc.cu -- split-precision (BF16x3) contraction on the Blackwell tensor
// cores: TMA -> shared memory -> tcgen05.mma (kind::f16, BF16 x BF16 -> FP32
// in TMEM) -> tcgen05.ld epilogue with FP64 alpha/beta.
//
// Each FP64 operand x is stored as two BF16 planes, hi = bf16(x) and
// lo = bf16(x - hi).  The kernel accumulates hi*hi + hi*lo + lo*hi for every
// K slice into one TMEM accumulator (the lo*lo term, ~2^-18 relative, is
// dropped), which gives ~16 significant bits per product and FP32 sums that
// are promoted to FP64 every CHUNK = 512 K elements (fewer for very long K).
//
// Persistent kernel, one CTA per SM, k tile 64 (128-byte swizzle):
//   warp 0  TMA producer (one elected lane)
//   warp 1  TMEM allocator + MMA issuer (one elected lane)
//   warps 2.. epilogue: two or three warps per TMEM lane quadrant, each
//             thread one output row x 48, 64 or 128 columns, accumulated in
//             FP64 across K chunks
// Three variants: one CTA per 128 x 144 output tile (14 warps, 3-stage
// mbarrier pipeline; the default), one CTA per 128 x 256 tile for launches
// whose tiles are single FP32-output chunks (10 warps, 2 stages), and for
// products of at least 256 rows a cluster pair of CTAs per 256 x 128 tile
// (tcgen05 cta_group::2, 10 warps, 4 stages), which halves each CTA's share
// of the B tile.  No copy uses cluster multicast.
// Every mbarrier wait is bounded by a %globaltimer limit; on expiry the
// kernel records an error code in g_tc_status, drains its own TMA copies,
// waits for its issued products, releases TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <mutex>
#include <unordered_map>

#include "common.cuh"
#include "gemm.cuh"

namespace acesb200 {

// hi = bf16(x) (round to nearest even), lo = bf16(x - hi); K padding is zero.
// Each thread converts two neighbouring K elements and stores them as one
// 32-bit BF16 pair per plane; Wide = false splits the pair index with FastDiv.
template <bool Wide>
__global__ void k_split_pack(__nv_bfloat162 *__restrict__ hi, __nv_bfloat162 *__restrict__ lo,
                             const double *__restrict__ src, long long ld, int k,
                             long long total_pairs, FastDiv fpairs) {
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total_pairs;
       idx += (long long)gridDim.x * blockDim.x) {
    long long r;
    int c;
    if (Wide) {
      r = idx / fpairs.d;
      c = 2 * (int)(idx - r * fpairs.d);
    } else {
      const unsigned q = fpairs.div((unsigned)idx);
      r = q;
      c = 2 * (int)((unsigned)idx - q * fpairs.d);
    }
    const double *row = src + r * ld;
    const double x0 = c < k ? row[c] : 0.0, x1 = c + 1 < k ? row[c + 1] : 0.0;
    __nv_bfloat16 h0, l0, h1, l1;
    split_bf16(x0, h0, l0);
    split_bf16(x1, h1, l1);
    hi[idx] = __halves2bfloat162(h0, h1);
    lo[idx] = __halves2bfloat162(l0, l1);
  }
}

int split_pack(SplitOperand &op, const double *src, long long ld, int rows, int k,
               cudaStream_t st) {
  int rp = rows;
  int kp = (k + kSplitKPad - 1) / kSplitKPad * kSplitKPad;
  size_t need = (size_t)rp * kp * 2 * 2;
  if (!op.hi || op.cap < need) {
    if (op.hi) dev_free(op.hi);
    op.hi = op.lo = nullptr;
    op.cap = 0;
    void *p = nullptr;
    if (dev_alloc((void **)&p, need) != cudaSuccess) {
      cudaGetLastError();
      set_error("split_pack: device allocation of %zu bytes failed", need);
      return ACES_ERR_NOMEM;
    }
    op.hi = p;
    op.cap = need;
  }
  op.rows = rows;
  op.k = k;
  op.rows_pad = rp;
  op.k_pad = kp;
  op.lo = (char *)op.hi + (size_t)rp * kp * 2;
  const long long pairs = (long long)rp * (kp / 2);
  long long nb = (pairs + 255) / 256;
  if (nb > 148 * 32) nb = 148 * 32;
  const FastDiv fp((unsigned)(kp / 2));
  if (pairs < (1LL << 31))
    k_split_pack<false><<<(unsigned)nb, 256, 0, st>>>(
        (__nv_bfloat162 *)op.hi, (__nv_bfloat162 *)op.lo, src, ld, k, pairs, fp);
  else
    k_split_pack<true><<<(unsigned)nb, 256, 0, st>>>(
        (__nv_bfloat162 *)op.hi, (__nv_bfloat162 *)op.lo, src, ld, k, pairs, fp);
  count_launch();
  ACES_CUDA(cudaGetLastError());
  return ACES_OK;
}

namespace {
// k tile: 64 BF16 (128-byte rows, 128-byte swizzle, 3 stages), or 32 BF16
// (64-byte rows, 64-byte swizzle), which fits 7 stages in shared memory but
// measured slower on B200 (packed ladder M = K = 16290, N = 400: 1.08 ms
// against 0.82 ms, tensor pipe 42 % against 57 % of active cycles).
#ifndef ACES_TC_TBK
#define ACES_TC_TBK 64
#endif
constexpr int TBM = 128, TBN = 128, TBK = ACES_TC_TBK;
// Tile width of the default one-CTA kernel: 144 columns (o^2 = 400 in three
// tiles, 3600 and 32400 in whole tiles, where 128-wide tiles leave a 16-wide
// remainder that costs nearly a full tile); TBN = 128 is the CTA-pair width.
#ifndef ACES_TC_NARROW
#define ACES_TC_NARROW 144
#endif
constexpr int TBN_1 = ACES_TC_NARROW;
static_assert(TBN_1 == 128 || TBN_1 == 144, "one-CTA tile width");
static_assert(TBK == 32 || TBK == 64, "k tile of 32 or 64 BF16");
constexpr int kRowBytes = TBK * 2;                    // one swizzled smem row
constexpr int kUnit = 64 / TBK;                       // k tiles per 64 K elements
constexpr int TILE_A = TBM * TBK * 2;                 // bytes of one BF16 plane tile of A
constexpr int kSmemLimit = 227 * 1024;
// Per-CTA pipeline geometry of the two variants: CG = 1, one CTA per 128 x 128
// output tile (A and B tiles of 128 rows); CG = 2, a CTA pair per 256 x 128
// tile (tcgen05 cta_group::2), each CTA holding its 128 rows of A and half of
// the B rows, so a k tile brings 48 KB per CTA into shared memory instead of
// 64 KB for the same products.
template <int CG, int BN = TBN>
struct Geom {
  static constexpr int kBRows = BN / CG;                    // B rows per CTA
  static constexpr int kTileB = kBRows * TBK * 2;
  static constexpr int kStage = 2 * TILE_A + 2 * kTileB;    // hi+lo of A and B
  static constexpr int kBarArea = 512;
  static constexpr int kStages = (kSmemLimit - 1024 - kBarArea) / kStage;
  static constexpr int kSmem = kStages * kStage + 1024 + kBarArea;  // + alignment + barriers
  static_assert(kSmem <= kSmemLimit && kStages >= (BN > 160 ? 2 : 3), "pipeline depth");
  static_assert(3 * kStages * 8 + 64 + 8 <= kBarArea, "barrier area");
};
// (3 stages at TBK 64 or 6/7 at TBK 32 for one CTA per tile, 4 at TBK 64 for
// pairs, 2 of 96 KB for the 128 x 256 tiles)
// k tiles per FP32 accumulation chunk, by the contraction length K: 512 K
// elements up to K = 36864, 256 up to 73728, 128 beyond
inline int chunk_for(int kTilesTotal) {
  if (kTilesTotal <= 576 * kUnit) return 8 * kUnit;
  if (kTilesTotal <= 1152 * kUnit) return 4 * kUnit;
  return 2 * kUnit;
}
// Epilogue warps of a tile width: 2 per TMEM lane quadrant (64 or 128 columns
// each), or 3 per quadrant for the 144-wide tiles (48 columns each, whose
// FP64 sums fit the registers of a 14-warp block)
template <int BN>
constexpr int epi_warps() { return BN % 64 == 0 ? 8 : 12; }
template <int BN>
constexpr int epi_cols() { return 4 * BN / epi_warps<BN>(); }  // columns per epilogue thread
template <int BN>
constexpr int block_threads() { return 32 * (2 + epi_warps<BN>()); }
static_assert(epi_cols<128>() == 64 && epi_cols<144>() == 48 && epi_cols<256>() == 128,
              "epilogue column spans");
// Wide tiles (128 x 256, one CTA): products whose every tile is a single
// accumulation chunk with FP32 output (the batched (T) classes) -- no FP64
// chunk sums to hold, so the epilogue streams the 256 TMEM columns straight
// to the output, and each tcgen05.mma carries N = 256 (half the instructions
// of the 128-wide tile for the same products).
constexpr int TBN_WIDE = 256;
#ifndef ACES_TC_WIDE
#define ACES_TC_WIDE 1
#endif
#ifndef ACES_TC_NACC
#define ACES_TC_NACC 2
#endif
constexpr int kNAcc = ACES_TC_NACC;                   // TMEM accumulators in rotation
template <int BN>
constexpr int tmem_cols() {  // a power of two >= 32 (allocation unit)
  int c = 32;
  while (c < kNAcc * BN) c *= 2;
  return c;
}
// Bound on every mbarrier wait (ns), per device; aces_set_wait_limit changes it.
__device__ unsigned long long g_tc_wait_ns = 4000000000ULL;
// Fault injection for tests of the bounded waits (aces_debug_inject): when set,
// the TMA producer issues no copies, so the MMA and epilogue waits run out,
// the kernel records a status and returns with nothing in flight.
__device__ int g_tc_inject = 0;

__device__ int g_tc_status;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// try_wait with a suspend-time hint: a waiting thread sleeps until the phase
// completes (or 20 us pass) instead of re-polling, which leaves the issue
// slots of its SM sub-partition to the MMA and TMA threads
#ifndef ACES_TC_HINT
#define ACES_TC_HINT 20000
#endif
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
#if ACES_TC_HINT > 0
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"((uint32_t)ACES_TC_HINT)
      : "memory");
#else
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
#endif
  return ok != 0;
}
// bounded wait: false on timeout
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = gtimer(), limit = g_tc_wait_ns;
  while (!mbar_try(bar, parity)) {
    if (gtimer() - t0 > limit) return false;
  }
  return true;
}
// cluster-scope forms for the CTA pair: waits that acquire at cluster scope
// (the phase is completed by arrivals of the other CTA), remote arrives,
// the partner's address of a shared variable, the cluster barrier
// (ACES_TC_CL_HINT: suspend-time hint of these waits in ns; 0 = none, the
// thread re-polls after the hardware's own short wait)
#ifndef ACES_TC_CL_HINT
#define ACES_TC_CL_HINT 20000
#endif
__device__ __forceinline__ bool mbar_try_cl(uint32_t bar, uint32_t parity) {
  uint32_t ok;
#if ACES_TC_CL_HINT > 0
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2, "
      "%3;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"((uint32_t)ACES_TC_CL_HINT)
      : "memory");
#else
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;"
      "\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
#endif
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_cl(uint32_t bar, uint32_t parity) {
  if (mbar_try_cl(bar, parity)) return true;
  const unsigned long long t0 = gtimer(), limit = g_tc_wait_ns;
  while (!mbar_try_cl(bar, parity)) {
    if (gtimer() - t0 > limit) return false;
  }
  return true;
}
// waits on barriers that the other CTA of a pair may complete (tcgen05
// commits multicast by rank 0, its copies, remote epilogue arrivals)
template <int CG>
__device__ __forceinline__ bool mbar_wait_g(uint32_t bar, uint32_t parity) {
  return CG == 2 ? mbar_wait_cl(bar, parity) : mbar_wait(bar, parity);
}
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t mapa_rank(uint32_t addr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr)
               : "memory");
}
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;" ::
                   : "memory");
}
// the same load issued by either CTA of a pair, completing on a barrier of
// rank 0 (shared::cluster address); the data lands in the issuing CTA
__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap *map, int x, int y,
                                                 uint32_t cluster_bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(cluster_bar)
      : "memory");
}
__device__ __forceinline__ void st_cluster_u32(uint32_t cluster_addr, uint32_t v) {
  asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(cluster_addr), "r"(v) : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
// UMMA shared-memory descriptor: K-major, swizzled rows of kRowBytes (128- or
// 64-byte swizzle, layout type 2 or 4), 8-row groups 8 * kRowBytes apart (SBO),
// LBO unused (1), sm100 descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)((8 * kRowBytes) >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)(kRowBytes == 128 ? 2 : 4) << 61;
  return d;
}
// instruction descriptor, kind::f16: D=F32, A=B=BF16, both K-major, N>>3, M>>4
// (the N field, bits 17-22, is set per tile: a ragged last n tile multiplies
// only its live columns rounded up to 16, the granularity of N at M = 128)
// (M = 128 per CTA: 128 for one CTA, 256 for a CTA pair)
constexpr uint32_t kIdescK = (1u << 4) | (1u << 7) | (1u << 10);
// MMA N of a tile with n_live live columns (multiple of 16, at most BN)
template <int BN = TBN>
__device__ __forceinline__ int mma_n(int n_live) { return min(BN, (n_live + 15) & ~15); }
template <int CG, int BN>
__device__ __forceinline__ uint32_t idesc_for(int n_live) {
  return kIdescK | ((uint32_t)((TBM * CG) >> 4) << 24) |
         ((uint32_t)(mma_n<BN>(n_live) >> 3) << 17);
}

template <int CG>
__device__ __forceinline__ void umma(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc,
                                     uint32_t acc) {
  if constexpr (CG == 1)
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
        "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
  else
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
        "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}
// completion of this thread's issued products arrives on `bar` (for a CTA
// pair: on the barrier at the same offset in both CTAs)
template <int CG>
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  if constexpr (CG == 1)
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
        : "memory");
  else
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
        " [%0], %1;" ::"r"(bar), "h"((unsigned short)3)
        : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t *r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
      "%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
      "%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}

// The MMA warp accumulates CHUNK K elements at a time in FP32 into one of two
// TMEM accumulators (ping-pong); the epilogue warps drain every finished chunk
// into FP64 registers while the next chunk is computed.  This bounds the number
// of FP32 tensor-core accumulations any partial sum sees to 3*CHUNK/16, so the
// truncation bias of the tensor-core adders stays small instead of growing
// with K.  The energy error of a CCSD solve grows linearly with CHUNK (o=20,
// v=180: 1.4e-8 Eh at 128, 2.7e-8 at 256, 5.3e-8 at 512) while the drain cost
// per product halves with every doubling; it also grows with the contraction
// length (o=30, v=270 with 512 throughout: 7.8e-7 Eh), so CHUNK is 512 up to
// K = 36864 and smaller beyond (chunk_for).
//
// The kernel is persistent: gridDim.x <= #SMs CTAs walk the output tiles
// t = blockIdx.x, blockIdx.x + gridDim.x, ... (the side with fewer tiles
// fastest, then the other, then the split-K slice z).  The TMA producer and
// the MMA issuer run their
// k-tile sequence straight across tile boundaries (stage and TMEM-buffer
// parities are global counters), so the loads and products of the next tile
// overlap the epilogue of the current one.
// One launch computes up to kMaxProb independent products (a grouped launch
// keeps every SM busy where one product has too few tiles for whole waves),
// each C_g = alpha * sum_s A_gs B_gs^T + beta C_g over up to kMaxSeg K
// segments with their own tensor maps.  Tiles are numbered problem by
// problem; within a problem as above.
constexpr int kMaxSeg = 4, kMaxProb = 3;
static_assert(kMaxSeg == kBatchSeg, "batch entries carry one row offset per segment");
struct Problem {
  CView C;
  int M, N, tilesM, tilesN;
  int ktc, kTilesTotal;  // k tiles per split-K slice, in total
  int tile0;             // first tile of this problem
  int mfast;             // tile order: m tile fastest (else n tile fastest)
  int nseg, chunk;
  int kt0[kMaxSeg + 1];  // segment s owns global k tiles [kt0[s], kt0[s+1])
  // batched problem: nbatch entries (row windows of the parents, output
  // offsets) in device memory, or nullptr
  const BatchEntry *batch;
  int nbatch;
  int f32out;            // output elements are FP32
};
struct Launch {
  CUtensorMap ah[kMaxProb][kMaxSeg], al[kMaxProb][kMaxSeg];
  CUtensorMap bh[kMaxProb][kMaxSeg], bl[kMaxProb][kMaxSeg];
  Problem prob[kMaxProb];
  int nprob, nTiles;
  int cg;  // CTAs per tile: 1, or 2 (a cluster pair on 256 x 128 tiles)
  int bn;  // tile width: TBN_1 (one CTA), TBN (CTA pair), TBN_WIDE (one CTA,
           // single-chunk FP32 output)
};
struct TileRef {
  int g, m0, n0, z, ktb, kTiles, b;
};
template <int CG, int BN>
__device__ __forceinline__ TileRef decode_tile(const Launch &L, int t) {
  TileRef r;
  r.g = 0;
  while (r.g + 1 < L.nprob && t >= L.prob[r.g + 1].tile0) ++r.g;
  const Problem &P = L.prob[r.g];
  const int tl = t - P.tile0;
  int tm, tn;
  r.b = 0;
  if (P.batch) {
    // fewer-tiles side fastest, then the entry, then the other side
    if (P.mfast) {
      tm = tl % P.tilesM;
      const int q = tl / P.tilesM;
      r.b = q % P.nbatch;
      tn = q / P.nbatch;
    } else {
      tn = tl % P.tilesN;
      const int q = tl / P.tilesN;
      r.b = q % P.nbatch;
      tm = q / P.nbatch;
    }
    r.z = 0;
  } else if (P.mfast) {
    tm = tl % P.tilesM;
    const int q = tl / P.tilesM;
    tn = q % P.tilesN;
    r.z = q / P.tilesN;
  } else {
    tn = tl % P.tilesN;
    const int q = tl / P.tilesN;
    tm = q % P.tilesM;
    r.z = q / P.tilesM;
  }
  r.m0 = tm * TBM * CG;
  r.n0 = tn * BN;
  r.ktb = r.z * P.ktc;
  r.kTiles = max(0, min(P.ktc, P.kTilesTotal - r.ktb));
  return r;
}

// row windows of a batched entry (one read per tile, 8 ints)
__device__ __forceinline__ void batch_rows(const Problem &P, int b, int (&rA)[kMaxSeg],
                                           int (&rB)[kMaxSeg]) {
  if (P.batch) {
    const int4 *e = reinterpret_cast<const int4 *>(P.batch + b);
    const int4 a = __ldg(e), c = __ldg(e + 1);
    rA[0] = a.x; rA[1] = a.y; rA[2] = a.z; rA[3] = a.w;
    rB[0] = c.x; rB[1] = c.y; rB[2] = c.z; rB[3] = c.w;
  } else {
#pragma unroll
    for (int q = 0; q < kMaxSeg; ++q) rA[q] = rB[q] = 0;
  }
}
// where k tile kt of tile T lies for this CTA: the K segment (tensor maps),
// the K offset, and the A and B row coordinates (this CTA's rows: A from
// m0 + 128 rank, B from n0 + rank * (MMA N) / 2)
struct StageAt {
  int sg, kx, ya, yb;
};
template <int CG, int BN>
__device__ __forceinline__ StageAt stage_at(const Problem &P, const TileRef &T,
                                            const int (&rA)[kMaxSeg], const int (&rB)[kMaxSeg],
                                            int kt, uint32_t rank) {
  const int gk = T.ktb + kt;
  int sg = 0;
  while (sg + 1 < P.nseg && gk >= P.kt0[sg + 1]) ++sg;
  StageAt s;
  s.sg = sg;
  s.kx = (gk - P.kt0[sg]) * TBK;
  s.ya = T.m0 + (int)rank * TBM;
  s.yb = T.n0 + (CG == 2 ? (int)rank * (mma_n<BN>(P.N - T.n0) >> 1) : 0);
#pragma unroll
  for (int q = 0; q < kMaxSeg; ++q)
    if (q == sg) {
      s.ya += rA[q];
      s.yb += rB[q];
    }
  return s;
}

// Epilogue of the wide tiles (one accumulation chunk per tile, FP32 output):
// each thread loads its row's 128 columns from TMEM (four 32-column loads),
// hands the buffer back to the MMA thread, then writes them: plain stores for
// beta = 0, one RED per element for beta = 1 (every element has one owner,
// so the sum equals load + add + store).  Same arithmetic as the chunked
// epilogue: (float)(alpha * (double)acc).
template <int CG, int BN>
__device__ __forceinline__ void epilogue_wide(const Launch &L, int t0, int tstep, uint32_t tmem,
                                              uint64_t *acc_full, uint64_t *acc_empty,
                                              int *abort_flag, double alpha, double beta,
                                              int q, int half, int lane) {
  constexpr int kC = epi_cols<BN>();  // columns per thread
  const int row = q * 32 + lane;
  int gc = 0;
  for (int t = t0; t < L.nTiles; t += tstep, ++gc) {
    const TileRef T = decode_tile<CG, BN>(L, t);
    const Problem &P = L.prob[T.g];
    const int b = gc % kNAcc;
    const bool w = mbar_wait_g<CG>(smem_u32(&acc_full[b]), (gc / kNAcc) & 1);
    if (!w) atomicExch(&g_tc_status, 4);
    if (!__all_sync(0xffffffffu, w && !*(volatile int *)abort_flag)) return;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int nb = T.n0 + half * kC;
    const int ncol = min(kC, P.N - nb);  // live columns (may be <= 0)
    const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BN + half * kC);
    uint32_t r[kC / 32][32];
#pragma unroll
    for (int h = 0; h < kC / 32; ++h)
      if (ncol > h * 32) tmem_ld32(tbase + h * 32, r[h]);  // warp-uniform condition
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_u32(&acc_empty[b]));
    const int m = T.m0 + row;
    if (m >= P.M || ncol <= 0) continue;
    const CView &C = P.C;
    float *const cm = reinterpret_cast<float *>(C.p) +
                      (P.batch ? __ldg(&P.batch[T.b].coff) : 0LL) +
                      cview_dim(C.mdiv, C.sm1, C.sm0, m);
    CViewNWalk wk(C, nb);
    float *const c0 = cm + wk.off;  // column nb
    if (beta == 0.0 && C.ndiv > 0x7fffffff && C.sn0 == 1 && ((uintptr_t)c0 & 15) == 0) {
      // unit n stride: the thread's columns are contiguous, 16-byte stores
#pragma unroll
      for (int h = 0; h < kC / 32; ++h)
#pragma unroll
        for (int j = 0; j < 32; j += 4) {
          const int c = h * 32 + j;
          float x[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) x[u] = (float)(alpha * (double)__uint_as_float(r[h][j + u]));
          if (c + 3 < ncol) {
            *reinterpret_cast<float4 *>(c0 + c) = make_float4(x[0], x[1], x[2], x[3]);
          } else {
#pragma unroll
            for (int u = 0; u < 4; ++u)
              if (c + u < ncol) c0[c + u] = x[u];
          }
        }
    } else if (beta == 0.0) {
#pragma unroll
      for (int h = 0; h < kC / 32; ++h)
#pragma unroll
        for (int j = 0; j < 32; ++j, wk.next())
          if (h * 32 + j < ncol) cm[wk.off] = (float)(alpha * (double)__uint_as_float(r[h][j]));
    } else {
#pragma unroll
      for (int h = 0; h < kC / 32; ++h)
#pragma unroll
        for (int j = 0; j < 32; ++j, wk.next())
          if (h * 32 + j < ncol)
            atomicAdd(cm + wk.off, (float)(alpha * (double)__uint_as_float(r[h][j])));
    }
  }
}

// One CTA per SM: registers are allocated per SM sub-partition (16384 each);
// with 10 warps three share one, so a thread gets at most 168 (the 128-wide
// epilogue spills a few of its 64 FP64 column sums, L1-resident), with 14
// warps four share one: 128 (the 144-wide epilogue's 48 sums fit, with a few
// spilled temporaries).
//
// CG = 2: clusters of two CTAs (ranks 0 and 1) share 256 x 128 tiles.  Each
// CTA's producer loads its 128 A rows and its half of the B rows (as many as
// the tile's MMA N needs: rows n0 + rank * N/2 on) into its own shared memory;
// all copies of a stage complete on rank 0's `full` barrier, which rank 0's
// producer arms with both CTAs' bytes, and warp 1 of rank 0 issues the
// cta_group::2 products (reading both CTAs' tiles) when it completes.
// Product completion is multicast to both CTAs' `empty`, `acc_full` and
// `mma_done` barriers; both CTAs' epilogues drain their own TMEM rows and
// arrive on rank 0's `acc_empty`.  Teardown: rank 1 reports how many stages
// it issued; after a cluster barrier rank 0 arms and waits out (bounded)
// any of them it did not arm itself (only after a wait gave up), so neither
// CTA leaves while a copy of the pair is in flight.
//
// BN = 256 (one CTA, 128 x 256 tiles): the launch's every tile is a single
// accumulation chunk with FP32 output; the epilogue streams each thread's 128
// TMEM columns to the output (two stages of 96 KB in shared memory).
template <int CG, int BN>
__global__ void __launch_bounds__(block_threads<BN>(), 1)
    k_gemm_bf16x3(const __grid_constant__ Launch L, double alpha, double beta,
                  double *__restrict__ part) {
  static_assert((CG == 2 && BN == TBN) || (CG == 1 && (BN == TBN_1 || BN == TBN_WIDE)),
                "tile variants");
  constexpr int kEpiWarps = epi_warps<BN>(), kCols = epi_cols<BN>();
  constexpr int kPiece = kCols % 32 == 0 ? 32 : 16;  // columns per TMEM load
  using Gm = Geom<CG, BN>;
  constexpr int kTmemCols = tmem_cols<BN>();
  constexpr int kStages = Gm::kStages, kStage = Gm::kStage, kTileB = Gm::kTileB;
  const int nTiles = L.nTiles;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + kStages * kStage);
  uint64_t *full = bars;                               // [kStages] TMA -> MMA (own copies)
  uint64_t *empty = bars + kStages;                    // [kStages] MMA -> TMA
  uint32_t *peer_issued = reinterpret_cast<uint32_t *>(bars + 2 * kStages);  // rank 1's stages
  uint64_t *acc_full = bars + 3 * kStages;             // [kNAcc] MMA -> epilogue
  uint64_t *acc_empty = acc_full + kNAcc;              // [kNAcc] epilogue -> MMA
  uint64_t *mma_done = acc_full + 2 * kNAcc;           // all products retired (teardown)
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mma_done + 1);
  int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = CG == 2 ? cluster_rank() : 0u;
  // tile walk: by CTA (CG = 1) or by CTA pair (CG = 2)
  const int t0 = CG == 2 ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
  const int tstep = CG == 2 ? (int)(gridDim.x >> 1) : (int)gridDim.x;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    for (int b = 0; b < kNAcc; ++b) {
      mbar_init(smem_u32(&acc_full[b]), 1);
      mbar_init(smem_u32(&acc_empty[b]), CG * kEpiWarps);
    }
    mbar_init(smem_u32(mma_done), 1);
    *abort_flag = 0;
    *peer_issued = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    if constexpr (CG == 1) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                       smem_u32(tmem_slot)),
                   "r"(kTmemCols));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    } else {
      asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                       smem_u32(tmem_slot)),
                   "r"(kTmemCols));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if constexpr (CG == 2) cluster_sync();  // both CTAs' barriers exist before any remote arrive
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer (every CTA: its own tiles) ----------------
    int it = 0;  // k tiles issued by this CTA
    bool stop = *(volatile int *)&g_tc_inject != 0;  // injected fault: issue nothing
    for (int t = t0; t < nTiles && !stop; t += tstep) {
      const TileRef T = decode_tile<CG, BN>(L, t);
      const Problem &P = L.prob[T.g];
      const int kTiles = T.kTiles;
      int rA[kMaxSeg], rB[kMaxSeg];
      batch_rows(P, T.b, rA, rB);
      for (int kt = 0; kt < kTiles; ++kt) {
        const int s = it % kStages;
        if (it >= kStages && !mbar_wait_g<CG>(smem_u32(&empty[s]), ((it / kStages) - 1) & 1)) {
          atomicExch(&g_tc_status, 1);
          *(volatile int *)abort_flag = 1;
          stop = true;
          break;
        }
        if (*(volatile int *)abort_flag) {
          stop = true;
          break;
        }
        const uint32_t fb = smem_u32(&full[s]);
        unsigned char *st = smem + s * kStage;
        // a pair's stage completes on rank 0's barrier, armed with both halves
        if (rank == 0) mbar_expect_tx(fb, CG * kStage);
        const StageAt sa = stage_at<CG, BN>(P, T, rA, rB, kt, rank);
        const int sg = sa.sg, kx = sa.kx, ya = sa.ya, yb = sa.yb;
        if (CG == 1) {
          tma_load_2d(smem_u32(st), &L.ah[T.g][sg], kx, ya, fb);
          tma_load_2d(smem_u32(st + TILE_A), &L.al[T.g][sg], kx, ya, fb);
          tma_load_2d(smem_u32(st + 2 * TILE_A), &L.bh[T.g][sg], kx, yb, fb);
          tma_load_2d(smem_u32(st + 2 * TILE_A + kTileB), &L.bl[T.g][sg], kx, yb, fb);
        } else {
          const uint32_t fb0 = mapa_rank(fb, 0);
          tma_load_2d_pair(smem_u32(st), &L.ah[T.g][sg], kx, ya, fb0);
          tma_load_2d_pair(smem_u32(st + TILE_A), &L.al[T.g][sg], kx, ya, fb0);
          tma_load_2d_pair(smem_u32(st + 2 * TILE_A), &L.bh[T.g][sg], kx, yb, fb0);
          tma_load_2d_pair(smem_u32(st + 2 * TILE_A + kTileB), &L.bl[T.g][sg], kx, yb, fb0);
        }
        ++it;
      }
    }
    if (rank == 0) {
      // drain: the most recent phase of every stage still possibly in flight
      const int first = it > kStages ? it - kStages : 0;
      for (int k = first; k < it; ++k)
        if (!mbar_wait_g<CG>(smem_u32(&full[k % kStages]), (k / kStages) & 1))
          atomicExch(&g_tc_status, 2);
      *(volatile int *)&peer_issued[1] = it;  // the stages this CTA armed
    } else {
      // rank 0 accounts for this CTA's copies at teardown
      st_cluster_u32(mapa_rank(smem_u32(peer_issued), 0), (uint32_t)it);
    }
  } else if (warp == 1 && lane == 0 && rank == 1) {
    // rank 1 issues no products: its TMEM is released after rank 0's last one
    if (!mbar_wait_g<CG>(smem_u32(mma_done), 0)) atomicExch(&g_tc_status, 6);
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer (rank 0) ----------------
    int it = 0, gc = 0;  // k tiles consumed, accumulation chunks started
    bool stop = false;
    for (int t = t0; t < nTiles && !stop; t += tstep) {
      const TileRef T = decode_tile<CG, BN>(L, t);
      const int kTiles = T.kTiles, chunk = L.prob[T.g].chunk;
      const uint32_t idesc = idesc_for<CG, BN>(L.prob[T.g].N - T.n0);
      for (int kt = 0; kt < kTiles; ++kt) {
        const int kin = kt % chunk, b = gc % kNAcc;
        if (kin == 0 && gc >= kNAcc &&
            !mbar_wait_g<CG>(smem_u32(&acc_empty[b]), ((gc / kNAcc) - 1) & 1)) {
          atomicExch(&g_tc_status, 5);
          *(volatile int *)abort_flag = 1;
          stop = true;
          break;
        }
        const int s = it % kStages;
        if (!mbar_wait_g<CG>(smem_u32(&full[s]), (it / kStages) & 1)) {
          atomicExch(&g_tc_status, 3);
          *(volatile int *)abort_flag = 1;
          stop = true;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t base = smem_u32(smem + s * kStage);
        const uint32_t ah = base, al = base + TILE_A, bh = base + 2 * TILE_A, bl = bh + kTileB;
        const uint32_t acc_t = tmem + (uint32_t)(b * BN);
        // the start address is the descriptor's low field (address >> 4): the
        // 32-byte K step (16 BF16) inside a swizzled row adds 2 to it
        const uint64_t dah = umma_desc(ah), dal = umma_desc(al), dbh = umma_desc(bh),
                       dbl = umma_desc(bl);
#pragma unroll
        for (int kk = 0; kk < TBK / 16; ++kk) {
          const uint64_t o = 2 * kk;
          const uint32_t acc = (kin > 0 || kk > 0) ? 1u : 0u;
          umma<CG>(acc_t, dah + o, dbh + o, idesc, acc);
          umma<CG>(acc_t, dah + o, dbl + o, idesc, 1u);
          umma<CG>(acc_t, dal + o, dbh + o, idesc, 1u);
        }
        umma_commit<CG>(smem_u32(&empty[s]));
        ++it;
        if (kin == chunk - 1 || kt == kTiles - 1) {
          umma_commit<CG>(smem_u32(&acc_full[b]));
          ++gc;
        }
      }
    }
    // every product issued by this thread has retired before TMEM is released
    umma_commit<CG>(smem_u32(mma_done));
    if (!mbar_wait_g<CG>(smem_u32(mma_done), 0)) atomicExch(&g_tc_status, 6);
  } else if (warp >= 2) {
    // ---------------- epilogue: FP64 accumulation of the chunks ----------------
    const int q = warp & 3;                 // TMEM lane quadrant accessible to this warp
    const int half = (warp - 2) >> 2;      // which kCols accumulator columns (0 .. kEpiWarps/4-1)
    const int row = q * 32 + lane;
    int gc = 0;
    bool ok = true;
    if constexpr (BN == TBN_WIDE)
      epilogue_wide<CG, BN>(L, t0, tstep, tmem, acc_full, acc_empty, abort_flag, alpha, beta, q,
                            half, lane);
    for (int t = t0; t < nTiles && ok && BN != TBN_WIDE; t += tstep) {
      const TileRef T = decode_tile<CG, BN>(L, t);
      const Problem &P = L.prob[T.g];
      const CView &C = P.C;
      const int M = P.M, N = P.N, m0 = T.m0 + (int)rank * TBM, n0 = T.n0, z = T.z;
      // lanes are consecutive output rows: with unit m stride a warp's stores coalesce
      const bool coalesced = C.sm0 == 1;
      const int nChunks = (T.kTiles + P.chunk - 1) / P.chunk;
      const int ncol = min(kCols, N - (n0 + half * kCols));  // live columns (may be <= 0)
      double acc[kCols];
#pragma unroll
      for (int j = 0; j < kCols; ++j) acc[j] = 0.0;
      for (int c = 0; c < nChunks; ++c, ++gc) {
        const int b = gc % kNAcc;
        const bool w = mbar_wait_g<CG>(smem_u32(&acc_full[b]), (gc / kNAcc) & 1);
        if (!w) atomicExch(&g_tc_status, 4);
        ok = __all_sync(0xffffffffu, w && !*(volatile int *)abort_flag);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t tbase =
            tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BN + half * kCols);
#pragma unroll
        for (int h = 0; h < kCols / kPiece; ++h) {
          if (ncol > h * kPiece) {  // warp-uniform: skip column groups past N
            uint32_t r[32];
            if constexpr (kPiece == 32)
              tmem_ld32(tbase + h * 32, r);
            else
              tmem_ld16(tbase + h * kPiece, r);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int j = 0; j < kPiece; ++j)
              acc[h * kPiece + j] += (double)__uint_as_float(r[j]);
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) {
          if constexpr (CG == 2)  // rank 0's barrier counts both CTAs' warps
            mbar_arrive_cluster(mapa_rank(smem_u32(&acc_empty[b]), 0));
          else
            mbar_arrive(smem_u32(&acc_empty[b]));
        }
      }
      if (!ok) break;
      const int m = m0 + row;
      if (m >= M || ncol <= 0) continue;
      const int nb = n0 + half * kCols;
      if (P.f32out) {
        // FP32 output (batched (T) W): plain stores for beta = 0, one RED per
        // element for beta = 1 (single owner, so it equals load + add + store)
        float *const cm = reinterpret_cast<float *>(C.p) +
                          (P.batch ? __ldg(&P.batch[T.b].coff) : 0LL) +
                          cview_dim(C.mdiv, C.sm1, C.sm0, m);
        CViewNWalk w(C, nb);
        if (beta == 0.0) {
#pragma unroll
          for (int j = 0; j < kCols; ++j, w.next())
            if (j < ncol) cm[w.off] = (float)(alpha * acc[j]);
        } else {
#pragma unroll
          for (int j = 0; j < kCols; ++j, w.next())
            if (j < ncol) atomicAdd(cm + w.off, (float)(alpha * acc[j]));
        }
      } else if (part) {
        // split-K partial, [z][n][m]: lanes write consecutive m
        double *pz = part + (size_t)z * M * N + m;
#pragma unroll
        for (int j = 0; j < kCols; ++j)
          if (j < ncol) pz[(size_t)(nb + j) * M] = acc[j];
      } else {
        double *const cm = C.p + (P.batch ? __ldg(&P.batch[T.b].coff) : 0LL) +
                           cview_dim(C.mdiv, C.sm1, C.sm0, m);
        CViewNWalk w(C, nb);
        if (beta == 0.0) {
#pragma unroll
          for (int j = 0; j < kCols; ++j, w.next())
            if (j < ncol) cm[w.off] = alpha * acc[j];
        } else if (beta == 1.0 && coalesced) {
          // one fire-and-forget FP64 add per element (RED): every element has a
          // single owner thread, so the result equals load + add + store
#pragma unroll
          for (int j = 0; j < kCols; ++j, w.next())
            if (j < ncol) atomicAdd(cm + w.off, alpha * acc[j]);
        } else {
          // read-modify-write in batches of 8: all loads of a batch are issued
          // before its stores, so the memory latency is paid once per batch
#pragma unroll
          for (int j0 = 0; j0 < kCols; j0 += 8) {
            double old[8];
            long long off[8];
#pragma unroll
            for (int j = 0; j < 8; ++j, w.next()) {
              off[j] = w.off;
              old[j] = j0 + j < ncol ? __ldg(cm + off[j]) : 0.0;
            }
#pragma unroll
            for (int j = 0; j < 8; ++j)
              if (j0 + j < ncol) cm[off[j]] = alpha * acc[j0 + j] + beta * old[j];
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if constexpr (CG == 2) {
    cluster_sync();  // rank 1's count of issued stages is in peer_issued[0]
    if (rank == 0 && threadIdx.x == 0) {
      // stages rank 1 issued that this CTA never armed (possible only after
      // a wait gave up): arm them with rank 1's bytes and wait them out
      const int mine = (int)*(volatile uint32_t *)&peer_issued[1];
      const int theirs = (int)*(volatile uint32_t *)&peer_issued[0];
      for (int k = mine; k < theirs; ++k) {
        const uint32_t fb = smem_u32(&full[k % kStages]);
        mbar_expect_tx(fb, kStage);
        if (!mbar_wait_g<CG>(fb, (k / kStages) & 1)) atomicExch(&g_tc_status, 8);
      }
    }
    __syncthreads();
    // a CTA of a pair leaves only when no copy, product or arrive of the pair
    // can still reach its shared memory
    cluster_sync();
  }
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if constexpr (CG == 1)
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                   "r"(kTmemCols));
    else
      asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                   "r"(kTmemCols));
  }
}

// multiprocessor count of the current device (persistent grid size)
int num_sms() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
      n = 148;
    cached[dev] = n;
  }
  return cached[dev];
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// Encoded maps by their only variable inputs: a map is a pure function of
// (address, rows, k, box rows), so a cached map is exactly what a new encode
// would produce, even for a freed and reused address.  (T) asks for the same
// operand views for every triplet: 16 maps per launch without the cache.
struct MapKey {
  const void *base;
  int rows_pad, k_pad, k, box_rows;
  bool operator==(const MapKey &o) const {
    return base == o.base && rows_pad == o.rows_pad && k_pad == o.k_pad && k == o.k &&
           box_rows == o.box_rows;
  }
};
struct MapKeyHash {
  size_t operator()(const MapKey &k) const {
    size_t h = std::hash<const void *>()(k.base);
    h ^= ((size_t)k.rows_pad * 0x9E3779B97F4A7C15ULL) + ((size_t)k.k_pad << 20) +
         ((size_t)k.k << 40) + k.box_rows;
    return h;
  }
};
struct MapCache {
  std::mutex mu;
  std::unordered_map<MapKey, CUtensorMap, MapKeyHash> maps;
};
MapCache &map_cache() {
  static MapCache *c = new MapCache();
  return *c;
}

// The map's K extent is the operand's true K (rows stay k_pad elements apart):
// the tail of the last k tile of a segment is the TMA's zero fill, read from
// neither L2 nor DRAM (for a K = nocc segment, 20 of the 64 columns of a k
// tile are data).  The padding in memory is zero as well, so the products
// are the same either way.
int make_map(CUtensorMap *m, void *base, int rows_pad, int k_pad, int k, int box_rows) {
  const MapKey key{base, rows_pad, k_pad, k, box_rows};
  MapCache &mc = map_cache();
  {
    std::lock_guard<std::mutex> lk(mc.mu);
    auto it = mc.maps.find(key);
    if (it != mc.maps.end()) {
      *m = it->second;
      return ACES_OK;
    }
  }
  EncodeTiledFn fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return ACES_ERR_CUDA;
  }
  cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows_pad};
  cuuint64_t strides[1] = {(cuuint64_t)k_pad * 2};
  cuuint32_t box[2] = {(cuuint32_t)TBK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE,
                  kRowBytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
    return ACES_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lk(mc.mu);
  if (mc.maps.size() >= 16384) mc.maps.clear();
  mc.maps.emplace(key, *m);
  return ACES_OK;
}
}  // namespace

namespace {
// fills problem g of a launch (maps, dims, chunk); tiles and split-K are set by the caller
int set_problem(Launch &L, int g, const SplitOperand *A, const SplitOperand *B, int nseg, int M,
                int N, const CView &C) {
  const int cg = L.cg == 2 ? 2 : 1;
  const int bn = cg == 2 ? TBN : (L.bn == TBN_WIDE ? TBN_WIDE : TBN_1);
  if (nseg < 1 || nseg > kMaxSeg) {
    set_error("gemm_nt_bf16x3: %d K segments (1..%d)", nseg, kMaxSeg);
    return ACES_ERR_ARG;
  }
  Problem &P = L.prob[g];
  P.C = C;
  P.M = M;
  P.N = N;
  P.nseg = nseg;
  P.kt0[0] = 0;
  for (int s = 0; s < nseg; ++s) {
    const SplitOperand &a = A[s], &b = B[s];
    if (a.k_pad != b.k_pad || a.rows < M || b.rows < N || a.k_pad % TBK || a.rows_pad < M ||
        b.rows_pad < N || a.k_pad == 0) {
      set_error("gemm_nt_bf16x3: operand shapes of segment %d do not match (%d/%d, %d, %d)", s,
                a.k_pad, b.k_pad, a.rows, b.rows);
      return ACES_ERR_ARG;
    }
    const int kk = std::min(a.k, b.k) > 0 ? std::min(a.k, b.k) : a.k_pad;
    ACES_TRY(make_map(&L.ah[g][s], a.hi, a.rows_pad, a.k_pad, kk, TBM));
    ACES_TRY(make_map(&L.al[g][s], a.lo, a.rows_pad, a.k_pad, kk, TBM));
    ACES_TRY(make_map(&L.bh[g][s], b.hi, b.rows_pad, b.k_pad, kk, bn / cg));
    ACES_TRY(make_map(&L.bl[g][s], b.lo, b.rows_pad, b.k_pad, kk, bn / cg));
    P.kt0[s + 1] = P.kt0[s] + a.k_pad / TBK;
  }
  for (int s = nseg + 1; s <= kMaxSeg; ++s) P.kt0[s] = P.kt0[nseg];
  P.kTilesTotal = P.kt0[nseg];
  P.ktc = P.kTilesTotal;
  P.chunk = chunk_for(P.kTilesTotal);
  P.tilesM = (M + TBM * cg - 1) / (TBM * cg);
  P.tilesN = (N + bn - 1) / bn;
  // the side with fewer tiles runs fastest, so the CTAs working at the same
  // time share the row block of the larger operand (read from DRAM once,
  // then from L2): with a few m tiles and many n tiles, B is the large operand
  P.mfast = P.tilesM < P.tilesN ? 1 : 0;
  return ACES_OK;
}

// CTA pairs the device keeps resident at once (the pair variant's grid is
// twice that, at most the SM count)
int max_pairs() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return num_sms() / 2;
  if (!cached[dev]) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)(num_sms() & ~1));
    cfg.blockDim = dim3(block_threads<TBN>());
    cfg.dynamicSmemBytes = Geom<2>::kSmem;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_gemm_bf16x3<2, TBN>, &cfg) != cudaSuccess ||
        n <= 0) {
      cudaGetLastError();
      n = num_sms() / 2;
    }
    cached[dev] = std::min(n, num_sms() / 2);
  }
  return cached[dev];
}

// The pair variant passes the same tests as the 1-CTA kernel, but on B200 it
// measured slower on the shapes that matter here (packed ladder of the
// o = 20, v = 180 cycle: 1.72 ms against 1.47 ms; (T) classes of o = 6,
// v = 128: 420 us against 404 us per launch), so it is off by default;
// aces_set_tc_pairs(1) turns it on for launches whose every problem has at
// least 256 rows (the height of its tiles).
std::atomic<int> g_tc_pairs{0};
bool pairs_for(int min_rows) { return g_tc_pairs.load() != 0 && min_rows >= 2 * TBM; }
// wide tiles for the single-chunk FP32-output launches (aces_set_tc_wide)
std::atomic<int> g_tc_wide{ACES_TC_WIDE};

int launch_prepared(Launch &L, double alpha, double beta, double *part, cudaStream_t st) {
  // the shared-memory opt-in and the status word are per device
  static bool attr[64] = {false};
  int dev = 0;
  ACES_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("gemm_nt_bf16x3: device %d outside 0..63", dev);
    return ACES_ERR_ARG;
  }
  if (!attr[dev]) {
    ACES_CUDA(cudaFuncSetAttribute(k_gemm_bf16x3<1, TBN_1>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   Geom<1, TBN_1>::kSmem));
    ACES_CUDA(cudaFuncSetAttribute(k_gemm_bf16x3<2, TBN>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, Geom<2>::kSmem));
    ACES_CUDA(cudaFuncSetAttribute(k_gemm_bf16x3<1, TBN_WIDE>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   Geom<1, TBN_WIDE>::kSmem));
    int zero = 0;
    ACES_CUDA(cudaMemcpyToSymbol(g_tc_status, &zero, sizeof(int)));
    attr[dev] = true;
  }
  if (L.cg == 2) {
    const unsigned pairs = (unsigned)std::max(1, std::min(L.nTiles, max_pairs()));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(2 * pairs);
    cfg.blockDim = dim3(block_threads<TBN>());
    cfg.dynamicSmemBytes = Geom<2>::kSmem;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    ACES_CUDA(cudaLaunchKernelEx(&cfg, k_gemm_bf16x3<2, TBN>, L, alpha, beta, part));
  } else if (L.bn == TBN_WIDE) {
    const unsigned grid = (unsigned)std::min(L.nTiles, num_sms());
    k_gemm_bf16x3<1, TBN_WIDE>
        <<<grid, block_threads<TBN_WIDE>(), Geom<1, TBN_WIDE>::kSmem, st>>>(L, alpha, beta,
                                                                             part);
  } else {
    const unsigned grid = (unsigned)std::min(L.nTiles, num_sms());
    k_gemm_bf16x3<1, TBN_1>
        <<<grid, block_threads<TBN_1>(), Geom<1, TBN_1>::kSmem, st>>>(L, alpha, beta, part);
  }
  count_launch();
  ACES_CUDA(cudaGetLastError());
  return ACES_OK;
}
}  // namespace

namespace {
// ---- tile autotuner -------------------------------------------------------
// With aces_set_autotune(1), the first product of each shape class on a
// device times the tile variants that apply to it and caches the fastest;
// later products of the class launch the cached variant directly.  Variants:
// one CTA per 128 x TBN_1 tile or CTA pairs (single and grouped products of
// >= 256 rows), split K at the wave-efficiency slice count or none (single
// products), and for batched FP32-output launches 128 x TBN_1 or 128 x 256
// tiles.  A class is the launch
// kind, the K segment (or problem) count, FP32 output, eligibility for pairs,
// and the output tile counts and k tile count rounded to two significant
// bits.  Each candidate runs once untimed and three times timed (CUDA events)
// on the product's stream, into the product's own output when beta = 0 and
// into a zeroed scratch array with unit m stride otherwise (the layout whose
// epilogue stores coalesce, which the dispatcher gives real outputs);
// batched launches with beta != 0 are
// not tuned (they take a cached choice or the default).  Nothing is tuned
// while the stream is being captured.  Every variant meets the same error
// bound (same K order and FP32 chunks); one replaces the default only when at
// least 3 % faster, so timing noise keeps the default.
struct TuneChoice {
  int cg = 1;       // CTAs per tile
  int bn = 0;       // batched FP32 output: tile width (0 = the default rule)
  int nosplit = 0;  // single products: 1 = no split K
  int changed = 0;  // cached entries: the choice differs from the built-in rule
};
struct TuneKey {
  int dev, kind, nseg, flags, tm, tn, kt;
  bool operator==(const TuneKey &o) const {
    return dev == o.dev && kind == o.kind && nseg == o.nseg && flags == o.flags &&
           tm == o.tm && tn == o.tn && kt == o.kt;
  }
};
struct TuneKeyHash {
  size_t operator()(const TuneKey &k) const {
    const int v[7] = {k.dev, k.kind, k.nseg, k.flags, k.tm, k.tn, k.kt};
    size_t h = 1469598103934665603ULL;
    for (int x : v) h = (h ^ (size_t)(unsigned)x) * 1099511628211ULL;
    return h;
  }
};
struct TuneState {
  std::mutex mu;
  std::unordered_map<TuneKey, TuneChoice, TuneKeyHash> cache;
  long long classes = 0, changed = 0;
  double ms = 0.0;  // device time spent in timed candidate runs
};
TuneState &tune_state() {
  static TuneState s;
  return s;
}
std::atomic<int> g_autotune{0};
// largest scratch output of a tuning run (larger products keep the default)
constexpr size_t kTuneScratchMax = size_t(1) << 30;

// x rounded to its two leading bits below the top one (4 classes per octave)
int bucket2(long long x) {
  if (x < 4) return (int)x;
  const int b = 63 - __builtin_clzll((unsigned long long)x);
  return (b << 2) | (int)((x >> (b - 2)) & 3);
}

bool tune_lookup(const TuneKey &key, TuneChoice *out) {
  TuneState &s = tune_state();
  std::lock_guard<std::mutex> lk(s.mu);
  auto it = s.cache.find(key);
  if (it == s.cache.end()) return false;
  *out = it->second;
  return true;
}
void tune_store(const TuneKey &key, const TuneChoice &ch, bool changed, double ms) {
  TuneState &s = tune_state();
  std::lock_guard<std::mutex> lk(s.mu);
  TuneChoice c = ch;
  c.changed = changed ? 1 : 0;
  if (s.cache.emplace(key, c).second) {
    ++s.classes;
    if (changed) ++s.changed;
    s.ms += ms;
  }
}
// whether candidates may be timed on st now (not while it is captured)
bool can_time(cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return cs == cudaStreamCaptureStatusNone;
}
// mean device ms of three runs after an untimed one
int time_runs(const std::function<int()> &run, cudaStream_t st, float *ms) {
  cudaEvent_t e[2] = {nullptr, nullptr};
  int rc = ACES_OK;
  for (int i = 0; i < 2 && rc == ACES_OK; ++i)
    if (cudaEventCreate(&e[i]) != cudaSuccess) {
      set_error("autotune: cudaEventCreate failed");
      rc = ACES_ERR_CUDA;
    }
  if (rc == ACES_OK) rc = run();
  if (rc == ACES_OK && cudaEventRecord(e[0], st) != cudaSuccess) rc = ACES_ERR_CUDA;
  for (int r = 0; r < 3 && rc == ACES_OK; ++r) rc = run();
  if (rc == ACES_OK && (cudaEventRecord(e[1], st) != cudaSuccess ||
                        cudaEventSynchronize(e[1]) != cudaSuccess ||
                        cudaEventElapsedTime(ms, e[0], e[1]) != cudaSuccess)) {
    set_error("autotune: event timing failed");
    rc = ACES_ERR_CUDA;
  }
  if (rc == ACES_OK) *ms /= 3.0f;
  for (int i = 0; i < 2; ++i)
    if (e[i]) cudaEventDestroy(e[i]);
  return rc;
}
// times the candidates (cands[0] = the default) with run(choice, scratch
// output or nullptr); returns the index of the one to keep
int tune_pick(const std::vector<TuneChoice> &cands,
              const std::function<int(const TuneChoice &)> &run, cudaStream_t st, int *pick,
              double *total_ms) {
  float t_def = 0.0f, best = 0.0f;
  *pick = 0;
  *total_ms = 0.0;
  for (size_t i = 0; i < cands.size(); ++i) {
    float ms = 0.0f;
    ACES_TRY(time_runs([&] { return run(cands[i]); }, st, &ms));
    *total_ms += 4.0 * ms;
    if (i == 0) {
      t_def = best = ms;
    } else if (ms < best) {
      best = ms;
      *pick = (int)i;
    }
  }
  if (*pick != 0 && best > 0.97f * t_def) *pick = 0;
  return ACES_OK;
}
// RAII scratch output of the tuning runs (zeroed, so accumulating trial runs
// read finite values)
struct TuneScratch {
  double *p = nullptr;
  ~TuneScratch() {
    if (p) dev_free(p);
  }
  int get(size_t doubles, cudaStream_t st) {
    if (dev_alloc((void **)&p, doubles * sizeof(double)) != cudaSuccess || !p) {
      p = nullptr;
      set_error("autotune: scratch allocation of %zu doubles failed", doubles);
      return ACES_ERR_NOMEM;
    }
    ACES_CUDA(cudaMemsetAsync(p, 0, doubles * sizeof(double), st));
    return ACES_OK;
  }
};

// split-K slice count of a single product: the count (at least 256 K elements
// each, at most ~4 waves of tiles) whose tiles fill the SMs' waves best, ties
// to fewer slices (less partial traffic); 1 when the tiles fill the SMs
int split_slices(long long tiles, int kTilesTotal, int nsm) {
  int Z = 1;
  if (tiles < nsm && kTilesTotal >= 8 * kUnit) {
    double best = 0.0;
    const long long zmax =
        std::min<long long>(kTilesTotal / (4 * kUnit), (4LL * nsm + tiles - 1) / tiles);
    for (int z = 2; z <= zmax; ++z) {
      const double waves = (double)(tiles * z) / nsm;
      const double eff = waves / std::ceil(waves);
      if (eff > best + 1e-9) {
        best = eff;
        Z = z;
      }
    }
  }
  return Z;
}

int multi_run(const TuneChoice &ch, const SplitOperand *A, const SplitOperand *B, int nseg,
              int M, int N, double alpha, double beta, const CView &C, cudaStream_t st) {
  Launch L;
  memset(&L, 0, sizeof(L));
  L.nprob = 1;
  L.cg = ch.cg == 2 ? 2 : 1;
  ACES_TRY(set_problem(L, 0, A, B, nseg, M, N, C));
  Problem &P = L.prob[0];
  // split K when the output has too few tiles to fill the SMs (CTA pairs)
  const long long tiles = (long long)P.tilesN * P.tilesM;
  const int nsm = L.cg == 2 ? max_pairs() : num_sms();
  int Z = ch.nosplit ? 1 : split_slices(tiles, P.kTilesTotal, nsm);
  double *part = nullptr;
  if (Z > 1) {
    P.ktc = (P.kTilesTotal + Z - 1) / Z;
    Z = (P.kTilesTotal + P.ktc - 1) / P.ktc;
    part = splitk_workspace((size_t)Z * M * N);
    if (!part) {
      set_error("gemm_nt_bf16x3: split-K workspace allocation failed");
      return ACES_ERR_NOMEM;
    }
  }
  const long long nTiles = tiles * Z;
  if (nTiles > (1LL << 31) - 1) {
    set_error("gemm_nt_bf16x3: %lld output tiles exceed the scheduler range", nTiles);
    return ACES_ERR_ARG;
  }
  P.tile0 = 0;
  L.nTiles = (int)nTiles;
  ACES_TRY(launch_prepared(L, alpha, beta, part, st));
  if (part) return splitk_reduce(C, part, M, N, Z, alpha, beta, st, true);
  return ACES_OK;
}

int grouped_run(int cg, const GroupedProblem *probs, int nprob, double alpha, double beta,
                cudaStream_t st) {
  Launch L;
  memset(&L, 0, sizeof(L));
  L.cg = cg == 2 ? 2 : 1;
  long long tiles = 0;
  int n = 0;
  for (int g = 0; g < nprob; ++g) {
    const GroupedProblem &q = probs[g];
    if (q.M <= 0 || q.N <= 0) continue;
    ACES_TRY(set_problem(L, n, q.A, q.B, q.nseg, q.M, q.N, q.C));
    L.prob[n].tile0 = (int)tiles;
    tiles += (long long)L.prob[n].tilesM * L.prob[n].tilesN;
    ++n;
  }
  if (n == 0) return ACES_OK;
  if (tiles > (1LL << 31) - 1) {
    set_error("gemm_nt_bf16x3_grouped: %lld output tiles exceed the scheduler range", tiles);
    return ACES_ERR_ARG;
  }
  L.nprob = n;
  L.nTiles = (int)tiles;
  return launch_prepared(L, alpha, beta, nullptr, st);
}

int batched_run(const TuneChoice &ch, const SplitOperand *Apar, const SplitOperand *Bpar,
                int nseg, int M, int N, const BatchEntry *d_entries, int nbatch, double alpha,
                double beta, const CView &C, bool f32out, cudaStream_t st) {
  Launch L;
  memset(&L, 0, sizeof(L));
  L.nprob = 1;
  L.cg = ch.cg == 2 ? 2 : 1;
  // FP32 output whose every tile is one accumulation chunk, with 144 < N <=
  // 256: one wide tile instead of a full and a ragged narrow one.  Where N
  // fits one narrow tile or is much larger, the 3-stage narrow tiles win
  // (o = 6, v = 128 class launches against 128-wide tiles: 32 % slower with
  // N = 128 on wide tiles, 3 % slower with N = 16384)
  if (L.cg == 2)
    L.bn = TBN;
  else if (ch.bn)
    L.bn = f32out ? ch.bn : TBN_1;
  else
    L.bn = f32out && N > TBN_1 && N <= TBN_WIDE && g_tc_wide.load() ? TBN_WIDE : TBN_1;
  ACES_TRY(set_problem(L, 0, Apar, Bpar, nseg, M, N, C));
  if (L.bn == TBN_WIDE && L.prob[0].kTilesTotal > L.prob[0].chunk) {
    L.bn = TBN_1;
    ACES_TRY(set_problem(L, 0, Apar, Bpar, nseg, M, N, C));
  }
  Problem &P = L.prob[0];
  P.batch = d_entries;
  P.nbatch = nbatch;
  P.f32out = f32out ? 1 : 0;
  const long long tiles = (long long)P.tilesM * P.tilesN * nbatch;
  if (tiles > (1LL << 31) - 1) {
    set_error("gemm_nt_bf16x3_batched: %lld output tiles exceed the scheduler range", tiles);
    return ACES_ERR_ARG;
  }
  P.tile0 = 0;
  L.nTiles = (int)tiles;
  return launch_prepared(L, alpha, beta, nullptr, st);
}

int current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return dev;
}
}  // namespace

int gemm_nt_bf16x3_multi(const SplitOperand *A, const SplitOperand *B, int nseg, int M, int N,
                         double alpha, double beta, const CView &C, cudaStream_t st) {
  if (M <= 0 || N <= 0) return ACES_OK;
  TuneChoice def;
  def.cg = pairs_for(M) ? 2 : 1;
  if (!g_autotune.load() || nseg < 1 || nseg > kMaxSeg)
    return multi_run(def, A, B, nseg, M, N, alpha, beta, C, st);
  int kt = 0;
  for (int s = 0; s < nseg; ++s) kt += A[s].k_pad / TBK;
  const long long tm = (M + TBM - 1) / TBM, tn = (N + TBN_1 - 1) / TBN_1;
  const TuneKey key{current_device(), 0, nseg, M >= 2 * TBM ? 1 : 0, bucket2(tm), bucket2(tn),
                    bucket2(kt)};
  TuneChoice ch;
  if (tune_lookup(key, &ch)) return multi_run(ch, A, B, nseg, M, N, alpha, beta, C, st);
  std::vector<TuneChoice> cands{def};
  if (def.cg == 1 && split_slices(tm * tn, kt, num_sms()) > 1) {
    TuneChoice c;
    c.nosplit = 1;
    cands.push_back(c);
  }
  if (M >= 2 * TBM) {
    TuneChoice c;
    c.cg = def.cg == 2 ? 1 : 2;
    cands.push_back(c);
  }
  const bool scratch_out = beta != 0.0;
  if (cands.size() == 1 || (scratch_out && (size_t)M * N * sizeof(double) > kTuneScratchMax)) {
    tune_store(key, def, false, 0.0);
    return multi_run(def, A, B, nseg, M, N, alpha, beta, C, st);
  }
  if (!can_time(st)) return multi_run(def, A, B, nseg, M, N, alpha, beta, C, st);
  int pick = 0;
  double ms = 0.0;
  {
    TuneScratch scr;
    CView Ct = C;
    if (scratch_out) {
      ACES_TRY(scr.get((size_t)M * N, st));
      Ct = cview_colmajor(scr.p, M);  // unit m stride, as the dispatcher arranges outputs
    }
    ACES_TRY(tune_pick(
        cands,
        [&](const TuneChoice &c) { return multi_run(c, A, B, nseg, M, N, alpha, beta, Ct, st); },
        st, &pick, &ms));
  }
  tune_store(key, cands[pick], pick != 0, ms);
  return multi_run(cands[pick], A, B, nseg, M, N, alpha, beta, C, st);
}

int gemm_nt_bf16x3_grouped(const GroupedProblem *probs, int nprob, double alpha, double beta,
                           cudaStream_t st) {
  if (nprob < 1 || nprob > kMaxProb) {
    set_error("gemm_nt_bf16x3_grouped: %d problems (1..%d)", nprob, kMaxProb);
    return ACES_ERR_ARG;
  }
  int min_rows = 1 << 30;
  long long tiles = 0, outs = 0;
  int kt = 0;
  for (int g = 0; g < nprob; ++g) {
    const GroupedProblem &q = probs[g];
    if (q.M <= 0 || q.N <= 0) continue;
    min_rows = std::min(min_rows, q.M);
    tiles += (long long)((q.M + TBM - 1) / TBM) * ((q.N + TBN_1 - 1) / TBN_1);
    outs += (long long)q.M * q.N;
    if (q.nseg >= 1 && q.nseg <= kMaxSeg)
      for (int s = 0; s < q.nseg; ++s) kt = std::max(kt, q.A[s].k_pad / TBK);
  }
  const int def = pairs_for(min_rows) ? 2 : 1;
  if (!g_autotune.load() || tiles == 0 || min_rows < 2 * TBM)
    return grouped_run(def, probs, nprob, alpha, beta, st);
  const TuneKey key{current_device(), 1, nprob, 1, bucket2(tiles), 0, bucket2(kt)};
  TuneChoice ch;
  if (tune_lookup(key, &ch)) return grouped_run(ch.cg, probs, nprob, alpha, beta, st);
  const bool scratch_out = beta != 0.0;
  if (scratch_out && (size_t)outs * sizeof(double) > kTuneScratchMax) {
    ch.cg = def;
    tune_store(key, ch, false, 0.0);
    return grouped_run(def, probs, nprob, alpha, beta, st);
  }
  if (!can_time(st)) return grouped_run(def, probs, nprob, alpha, beta, st);
  std::vector<TuneChoice> cands(2);
  cands[0].cg = def;
  cands[1].cg = def == 2 ? 1 : 2;
  int pick = 0;
  double ms = 0.0;
  {
    TuneScratch scr;
    GroupedProblem tp[kMaxProb];
    for (int g = 0; g < nprob; ++g) tp[g] = probs[g];
    if (scratch_out) {
      ACES_TRY(scr.get((size_t)outs, st));
      size_t off = 0;
      for (int g = 0; g < nprob; ++g) {
        if (tp[g].M <= 0 || tp[g].N <= 0) continue;
        tp[g].C = cview_colmajor(scr.p + off, tp[g].M);
        off += (size_t)tp[g].M * tp[g].N;
      }
    }
    ACES_TRY(tune_pick(
        cands, [&](const TuneChoice &c) { return grouped_run(c.cg, tp, nprob, alpha, beta, st); },
        st, &pick, &ms));
  }
  tune_store(key, cands[pick], pick != 0, ms);
  return grouped_run(cands[pick].cg, probs, nprob, alpha, beta, st);
}

int gemm_nt_bf16x3(const SplitOperand &A, const SplitOperand &B, int M, int N, double alpha,
                   double beta, const CView &C, cudaStream_t st) {
  return gemm_nt_bf16x3_multi(&A, &B, 1, M, N, alpha, beta, C, st);
}

int gemm_nt_bf16x3_batched(const SplitOperand *Apar, const SplitOperand *Bpar, int nseg, int M,
                           int N, const BatchEntry *h_entries, const BatchEntry *d_entries,
                           int nbatch, double alpha, double beta, const CView &C, bool f32out,
                           cudaStream_t st) {
  if (M <= 0 || N <= 0 || nbatch <= 0) return ACES_OK;
  if (f32out && beta != 0.0 && beta != 1.0) {
    set_error("gemm_nt_bf16x3_batched: FP32 output takes beta 0 or 1 (%g)", beta);
    return ACES_ERR_ARG;
  }
  if (f32out && C.sm0 != 1 && !(beta == 0.0 && C.sn0 == 1)) {
    set_error("gemm_nt_bf16x3_batched: FP32 output needs unit m stride (or n, for beta = 0)");
    return ACES_ERR_ARG;
  }
  if (nseg < 1 || nseg > kMaxSeg) {
    set_error("gemm_nt_bf16x3_batched: %d K segments (1..%d)", nseg, kMaxSeg);
    return ACES_ERR_ARG;
  }
  // every live row of every window inside its parent: the TMA coordinates of
  // live rows stay in range, rows past a window read its neighbours (or the
  // zero fill past the parent) and only reach discarded outputs
  for (int e = 0; e < nbatch; ++e)
    for (int s = 0; s < nseg; ++s) {
      const BatchEntry &q = h_entries[e];
      if (q.rowA[s] < 0 || (long long)q.rowA[s] + M > Apar[s].rows || q.rowB[s] < 0 ||
          (long long)q.rowB[s] + N > Bpar[s].rows || q.coff < 0) {
        set_error("gemm_nt_bf16x3_batched: entry %d segment %d outside its operands", e, s);
        return ACES_ERR_ARG;
      }
    }
  TuneChoice def;
  def.cg = pairs_for(M) ? 2 : 1;
  if (!g_autotune.load())
    return batched_run(def, Apar, Bpar, nseg, M, N, d_entries, nbatch, alpha, beta, C, f32out,
                       st);
  int kt = 0;
  for (int s = 0; s < nseg; ++s) kt += Apar[s].k_pad / TBK;
  const long long tm = (M + TBM - 1) / TBM, tn = (N + TBN_1 - 1) / TBN_1;
  const TuneKey key{current_device(), 2, nseg,
                    (M >= 2 * TBM ? 1 : 0) | (f32out ? 2 : 0) | (N > TBN_1 ? 4 : 0) |
                        (N > TBN_WIDE ? 8 : 0),
                    bucket2(tm * nbatch), bucket2(tn), bucket2(kt)};
  TuneChoice ch;
  if (tune_lookup(key, &ch))
    return batched_run(ch, Apar, Bpar, nseg, M, N, d_entries, nbatch, alpha, beta, C, f32out,
                       st);
  // the trial runs write the product's own output: only for beta = 0
  if (beta != 0.0 || !can_time(st))
    return batched_run(def, Apar, Bpar, nseg, M, N, d_entries, nbatch, alpha, beta, C, f32out,
                       st);
  // both widths of the one-CTA tile (cands[0] keeps the default rule); the
  // CTA pairs stay with the aces_set_tc_pairs switch here
  std::vector<TuneChoice> cands{def};
  if (def.cg == 1 && f32out && N > TBN_1 && N <= TBN_WIDE && kt <= chunk_for(kt)) {
    TuneChoice c;
    c.bn = g_tc_wide.load() ? TBN_1 : TBN_WIDE;
    cands.push_back(c);
  }
  if (cands.size() == 1) {
    tune_store(key, def, false, 0.0);
    return batched_run(def, Apar, Bpar, nseg, M, N, d_entries, nbatch, alpha, beta, C, f32out,
                       st);
  }
  int pick = 0;
  double ms = 0.0;
  ACES_TRY(tune_pick(cands,
                     [&](const TuneChoice &c) {
                       return batched_run(c, Apar, Bpar, nseg, M, N, d_entries, nbatch, alpha,
                                          beta, C, f32out, st);
                     },
                     st, &pick, &ms));
  tune_store(key, cands[pick], pick != 0, ms);
  return batched_run(cands[pick], Apar, Bpar, nseg, M, N, d_entries, nbatch, alpha, beta, C,
                     f32out, st);
}

void tc_set_autotune(int on) { g_autotune.store(on ? 1 : 0); }

void tc_autotune_reset() {
  TuneState &s = tune_state();
  std::lock_guard<std::mutex> lk(s.mu);
  s.cache.clear();
  s.classes = s.changed = 0;
  s.ms = 0.0;
}

void tc_autotune_stats(long long *classes, long long *changed, double *ms) {
  TuneState &s = tune_state();
  std::lock_guard<std::mutex> lk(s.mu);
  if (classes) *classes = s.classes;
  if (changed) *changed = s.changed;
  if (ms) *ms = s.ms;
}

// Text form of the current device's cached choices: a header line, then one
// line per class, "kind nseg flags tm tn kt cg bn nosplit changed", sorted.
static const char kTuneHeader[] = "# aces-b200 tile choices v1";

int tc_autotune_save(const char *path) {
  if (!path) {
    set_error("aces_autotune_save: null path");
    return ACES_ERR_ARG;
  }
  const int dev = current_device();
  std::vector<std::array<int, 10>> rows;
  {
    TuneState &s = tune_state();
    std::lock_guard<std::mutex> lk(s.mu);
    for (const auto &kv : s.cache)
      if (kv.first.dev == dev)
        rows.push_back({kv.first.kind, kv.first.nseg, kv.first.flags, kv.first.tm, kv.first.tn,
                        kv.first.kt, kv.second.cg, kv.second.bn, kv.second.nosplit,
                        kv.second.changed});
  }
  std::sort(rows.begin(), rows.end());
  FILE *f = fopen(path, "w");
  if (!f) {
    set_error("aces_autotune_save: cannot open %s for writing", path);
    return ACES_ERR_ARG;
  }
  fprintf(f, "%s\n", kTuneHeader);
  for (const auto &r : rows)
    fprintf(f, "%d %d %d %d %d %d %d %d %d %d\n", r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7],
            r[8], r[9]);
  if (fclose(f) != 0) {
    set_error("aces_autotune_save: write to %s failed", path);
    return ACES_ERR_ARG;
  }
  return ACES_OK;
}

int tc_autotune_load(const char *path) {
  if (!path) {
    set_error("aces_autotune_load: null path");
    return ACES_ERR_ARG;
  }
  FILE *f = fopen(path, "r");
  if (!f) {
    set_error("aces_autotune_load: cannot open %s", path);
    return ACES_ERR_ARG;
  }
  char line[256];
  int lineno = 0;
  std::vector<std::pair<TuneKey, TuneChoice>> rows;
  const int dev = current_device();
  int rc = ACES_OK;
  while (fgets(line, sizeof line, f)) {
    ++lineno;
    if (lineno == 1) {
      if (strncmp(line, kTuneHeader, sizeof kTuneHeader - 1) != 0) {
        set_error("aces_autotune_load: %s is not a tile-choice file", path);
        rc = ACES_ERR_ARG;
        break;
      }
      continue;
    }
    int v[10];
    char extra;
    const int n = sscanf(line, "%d %d %d %d %d %d %d %d %d %d %c", &v[0], &v[1], &v[2], &v[3],
                         &v[4], &v[5], &v[6], &v[7], &v[8], &v[9], &extra);
    const int kind = v[0], nseg = v[1], flags = v[2], cg = v[6], bn = v[7], nosplit = v[8],
              changed = v[9];
    // each choice must be one the tuner could have made for its class
    const bool ok =
        n == 10 && kind >= 0 && kind <= 2 && nseg >= 1 &&
        nseg <= (kind == 1 ? kMaxProb : kMaxSeg) && flags >= 0 && flags <= 15 && v[3] >= 0 &&
        v[4] >= 0 && v[5] >= 0 && (cg == 1 || (cg == 2 && (flags & 1))) &&
        (bn == 0 || (kind == 2 && (flags & 2) && cg == 1 && (bn == TBN_1 || bn == TBN_WIDE))) &&
        (nosplit == 0 || (nosplit == 1 && kind == 0 && cg == 1)) && (changed == 0 || changed == 1);
    if (!ok) {
      set_error("aces_autotune_load: %s line %d is not a valid tile choice", path, lineno);
      rc = ACES_ERR_ARG;
      break;
    }
    TuneChoice c;
    c.cg = cg;
    c.bn = bn;
    c.nosplit = nosplit;
    c.changed = changed;
    rows.push_back({TuneKey{dev, kind, nseg, flags, v[3], v[4], v[5]}, c});
  }
  fclose(f);
  if (rc == ACES_OK && lineno == 0) {
    set_error("aces_autotune_load: %s is empty", path);
    rc = ACES_ERR_ARG;
  }
  if (rc != ACES_OK) return rc;
  // all lines valid: replace the classes they name, recount
  TuneState &s = tune_state();
  std::lock_guard<std::mutex> lk(s.mu);
  for (const auto &r : rows) s.cache[r.first] = r.second;
  s.classes = (long long)s.cache.size();
  s.changed = 0;
  for (const auto &kv : s.cache) s.changed += kv.second.changed;
  return ACES_OK;
}

SplitOperand split_view(const SplitOperand &p, int row0, int rows) {
  SplitOperand v = p;
  size_t off = (size_t)row0 * p.k_pad * 2;
  v.hi = (char *)p.hi + off;
  v.lo = (char *)p.lo + off;
  v.rows = rows;
  v.rows_pad = std::min(rows, p.rows_pad - row0);  // beyond it the tensor map zero-fills
  v.cap = 0;
  return v;
}

int tc_set_wait_limit(unsigned long long ns) {
  ACES_CUDA(cudaMemcpyToSymbol(g_tc_wait_ns, &ns, sizeof(ns)));
  return ACES_OK;
}

void tc_set_pairs(int on) { g_tc_pairs.store(on ? 1 : 0); }

void tc_set_wide(int on) { g_tc_wide.store(on ? 1 : 0); }

bool bf16x3_wide_applies(const SplitOperand *A, int nseg, int N) {
  if (!g_tc_wide.load() || pairs_for(1 << 30) || N <= TBN_1 || N > TBN_WIDE || nseg < 1 ||
      nseg > kMaxSeg)
    return false;
  int kt = 0;
  for (int s = 0; s < nseg; ++s) kt += A[s].k_pad / TBK;
  return kt <= chunk_for(kt);
}

int tc_set_inject(int on) {
  ACES_CUDA(cudaMemcpyToSymbol(g_tc_inject, &on, sizeof(on)));
  return ACES_OK;
}

int tc_status_and_clear() {
  int v = 0, zero = 0;
  if (cudaMemcpyFromSymbol(&v, g_tc_status, sizeof(int)) != cudaSuccess) return -1;
  if (v) cudaMemcpyToSymbol(g_tc_status, &zero, sizeof(int));
  return v;
}

}  // namespace acesb200
