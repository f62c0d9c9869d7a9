// kernels.cu -- bandwidth-bound kernels of the CC engine: resorts, FTAU,
// NEWT2/E4SENG, CMPENG, DIIS reductions, the DIIS solve and DPD gathers.
#include <algorithm>
#include <cstdio>

#include "common.cuh"
#include "gemm.cuh"
#include "kernels.cuh"

namespace acesb200 {

// ---------------------------------------------------------------------------
// Resort: generic 4-index permute-accumulate.
// ---------------------------------------------------------------------------
struct PermArgs {
  int n[4];
  int nterms;
  const double *src[4];
  double alpha[4];
  long long s[4][4];
  double beta;
  FastDiv fd1, fd2, fd3;  // divisors n[1], n[2], n[3]
};

// two BF16 values as one 32-bit word, the first at the lower address
__device__ __forceinline__ unsigned pack_bf16x2(__nv_bfloat16 a, __nv_bfloat16 b) {
  return (unsigned)__bfloat16_as_ushort(a) | ((unsigned)__bfloat16_as_ushort(b) << 16);
}

// Optional BF16 split planes of a resort's output, read as a rows x K
// K-contiguous contraction operand: output element idx (below 2^31) is
// operand element (r, c) = (idx / K, idx % K), stored at r * k_pad + c of
// both planes (the K padding is zero from the planes' allocation).
struct SplitOut {
  __nv_bfloat16 *hi = nullptr, *lo = nullptr;
  int k_pad = 0;
  FastDiv fk;  // divisor K
};

__device__ __forceinline__ void put_split(const SplitOut &so, long long idx, double x) {
  const unsigned r = so.fk.div((unsigned)idx);
  const long long p = (long long)r * so.k_pad + ((unsigned)idx - r * so.fk.d);
  __nv_bfloat16 h, l;
  split_bf16(x, h, l);
  so.hi[p] = h;
  so.lo[p] = l;
}

// Wide = false: element count below 2^31, indices split with FastDiv.  S:
// the output also goes to split planes (out may then be null: no FP64 copy).
template <bool Wide, bool S>
__global__ void k_permute_naive(double *__restrict__ out, PermArgs a, long long total,
                                SplitOut so) {
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    int i0, i1, i2, i3;
    if (Wide) {
      long long r = idx;
      i3 = r % a.n[3]; r /= a.n[3];
      i2 = r % a.n[2]; r /= a.n[2];
      i1 = r % a.n[1]; r /= a.n[1];
      i0 = (int)r;
    } else {
      unsigned r = (unsigned)idx, q;
      q = a.fd3.div(r); i3 = (int)(r - q * a.fd3.d); r = q;
      q = a.fd2.div(r); i2 = (int)(r - q * a.fd2.d); r = q;
      q = a.fd1.div(r); i1 = (int)(r - q * a.fd1.d);
      i0 = (int)q;
    }
    double acc = a.beta == 0.0 ? 0.0 : a.beta * out[idx];
    for (int t = 0; t < a.nterms; ++t)
      acc += a.alpha[t] * __ldg(a.src[t] + i0 * a.s[t][0] + i1 * a.s[t][1] + i2 * a.s[t][2] +
                                i3 * a.s[t][3]);
    if (!S || out) out[idx] = acc;
    if (S) put_split(so, idx, acc);
  }
}

// The gather of k_permute_naive for outputs whose innermost extent is a
// multiple of 4 (every source has unit stride along it): a thread owns 4
// consecutive outputs of one row, splits its index once and issues 4
// independent loads per term and two 16-byte stores (with S and K % 4 == 0,
// one 8-byte store per split plane).
template <bool S>
__global__ void k_permute_rows4(double *__restrict__ out, PermArgs a, long long quads,
                                SplitOut so) {
  for (long long qd = blockIdx.x * (long long)blockDim.x + threadIdx.x; qd < quads;
       qd += (long long)gridDim.x * blockDim.x) {
    const long long idx = qd * 4;
    unsigned r = (unsigned)idx, q;
    q = a.fd3.div(r); const int i3 = (int)(r - q * a.fd3.d); r = q;
    q = a.fd2.div(r); const int i2 = (int)(r - q * a.fd2.d); r = q;
    q = a.fd1.div(r); const int i1 = (int)(r - q * a.fd1.d);
    const int i0 = (int)q;
    double acc[4];
    if (a.beta == 0.0) {
      acc[0] = acc[1] = acc[2] = acc[3] = 0.0;
    } else {
      const double2 o0 = *reinterpret_cast<const double2 *>(out + idx);
      const double2 o1 = *reinterpret_cast<const double2 *>(out + idx + 2);
      acc[0] = a.beta * o0.x; acc[1] = a.beta * o0.y;
      acc[2] = a.beta * o1.x; acc[3] = a.beta * o1.y;
    }
    for (int t = 0; t < a.nterms; ++t) {
      const double *src = a.src[t] + i0 * a.s[t][0] + i1 * a.s[t][1] + i2 * a.s[t][2] + i3;
      double x[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) x[u] = __ldg(src + u);
#pragma unroll
      for (int u = 0; u < 4; ++u) acc[u] += a.alpha[t] * x[u];
    }
    if (!S || out) {
      *reinterpret_cast<double2 *>(out + idx) = make_double2(acc[0], acc[1]);
      *reinterpret_cast<double2 *>(out + idx + 2) = make_double2(acc[2], acc[3]);
    }
    if (S) {
      if ((so.fk.d & 3u) == 0) {  // the 4 outputs are one aligned run of an operand row
        const unsigned rr = so.fk.div((unsigned)idx);
        const long long p = (long long)rr * so.k_pad + ((unsigned)idx - rr * so.fk.d);
        __nv_bfloat16 h[4], l[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) split_bf16(acc[u], h[u], l[u]);
        *reinterpret_cast<uint2 *>(so.hi + p) =
            make_uint2(pack_bf16x2(h[0], h[1]), pack_bf16x2(h[2], h[3]));
        *reinterpret_cast<uint2 *>(so.lo + p) =
            make_uint2(pack_bf16x2(l[0], l[1]), pack_bf16x2(l[2], l[3]));
      } else {
#pragma unroll
        for (int u = 0; u < 4; ++u) put_split(so, idx + u, acc[u]);
      }
    }
  }
}

// Shared-memory tiles of R (32 or 64) i3 x 32 i_d, where every term reads
// either i_d with unit stride (transposed through the tile: reads coalesced
// along i_d) or i3 with unit stride (read at the output positions directly);
// writes coalesced along i3.  A 32 x 8 thread block; each thread loads R/8
// elements per term (all issued before they are used) and writes R/8 outputs.
template <int D, bool S, int R>
__global__ void __launch_bounds__(256) k_permute_tiled(double *__restrict__ out, PermArgs a,
                                                       SplitOut so) {
  __shared__ double tile[32][R + 1];
  constexpr int kL = R / 8;  // loads per thread and term (rows i3 = ty + 8 k)
  const int nd = a.n[D];
  const int t3 = (a.n[3] + R - 1) / R, td = (nd + 31) / 32;
  long long b = blockIdx.x;
  int b3 = b % t3; b /= t3;
  int bd = b % td; b /= td;
  // remaining two dims (the ones that are neither 3 nor D)
  int o0 = -1, o1 = -1;
  for (int k = 0; k < 3; ++k)
    if (k != D) { if (o0 < 0) o0 = k; else o1 = k; }
  int io1 = b % a.n[o1];
  int io0 = (int)(b / a.n[o1]);
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  // outputs of this thread: i3 = b3*R + tx + 32 h, id = bd*32 + ty + 8 k
  double acc[R / 32][4];
#pragma unroll
  for (int h = 0; h < R / 32; ++h)
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[h][k] = 0.0;
  const int id_ld = bd * 32 + tx;
  bool tile_used = false;
  for (int t = 0; t < a.nterms; ++t) {
    const double *base = a.src[t] + (long long)io0 * a.s[t][o0] + (long long)io1 * a.s[t][o1];
    if (a.s[t][3] == 1) {
      // a term with unit stride along i3 reads the output's own positions:
      // coalesced along i3 without the shared-memory transpose
      double v[R / 32][4];
#pragma unroll
      for (int h = 0; h < R / 32; ++h)
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int i3 = b3 * R + tx + 32 * h, id = bd * 32 + ty + 8 * k;
          v[h][k] = (i3 < a.n[3] && id < nd) ? __ldg(base + i3 + (long long)id * a.s[t][D]) : 0.0;
        }
#pragma unroll
      for (int h = 0; h < R / 32; ++h)
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[h][k] += a.alpha[t] * v[h][k];
      continue;
    }
    const double *src = base + (long long)id_ld * a.s[t][D];
    double v[kL];
#pragma unroll
    for (int k = 0; k < kL; ++k) {
      const int i3 = b3 * R + ty + 8 * k;
      v[k] = (i3 < a.n[3] && id_ld < nd) ? __ldg(src + (long long)i3 * a.s[t][3]) : 0.0;
    }
    if (tile_used) __syncthreads();  // the previous transposed term's tile is consumed
#pragma unroll
    for (int k = 0; k < kL; ++k) tile[tx][ty + 8 * k] = v[k];
    __syncthreads();
    tile_used = true;
#pragma unroll
    for (int h = 0; h < R / 32; ++h)
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[h][k] += a.alpha[t] * tile[ty + 8 * k][tx + 32 * h];
  }
#pragma unroll
  for (int h = 0; h < R / 32; ++h)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int i3 = b3 * R + tx + 32 * h, id = bd * 32 + ty + 8 * k;
      if (i3 < a.n[3] && id < nd) {
        int idx_[4];
        idx_[3] = i3; idx_[D] = id; idx_[o0] = io0; idx_[o1] = io1;
        long long o =
            (((long long)idx_[0] * a.n[1] + idx_[1]) * a.n[2] + idx_[2]) * a.n[3] + idx_[3];
        const double val = (a.beta == 0.0 ? 0.0 : a.beta * out[o]) + acc[h][k];
        if (!S || out) out[o] = val;
        if (S) put_split(so, o, val);
      }
    }
}

template <bool S>
static void permute_launch(double *out, PermArgs &a, const PermSpec &spec, long long total,
                           const SplitOut &so, cudaStream_t st) {
  // tiled path when the innermost output index is strided in some source and
  // another index D has unit stride in every source that is strided along i3
  int D = -1;
  bool all_unit3 = true;
  for (int t = 0; t < spec.nterms; ++t)
    if (a.s[t][3] != 1) all_unit3 = false;
  if (!all_unit3) {
    for (int d = 0; d < 3 && D < 0; ++d) {
      bool ok = true;
      for (int t = 0; t < spec.nterms; ++t)
        if (a.s[t][d] != 1 && a.s[t][3] != 1) ok = false;
      if (ok && a.n[d] >= 8) D = d;
    }
  }
  if (D >= 0 && a.n[3] >= 8) {
    // 64-row tiles (8 loads in flight per thread and term) unless i3 is short
    const int R = a.n[3] >= 48 ? 64 : 32;
    long long nb = (long long)((a.n[3] + R - 1) / R) * ((a.n[D] + 31) / 32);
    for (int k = 0; k < 3; ++k)
      if (k != D) nb *= a.n[k];
    dim3 blk(32, 8);
    if (R == 64) {
      if (D == 0) k_permute_tiled<0, S, 64><<<(unsigned)nb, blk, 0, st>>>(out, a, so);
      if (D == 1) k_permute_tiled<1, S, 64><<<(unsigned)nb, blk, 0, st>>>(out, a, so);
      if (D == 2) k_permute_tiled<2, S, 64><<<(unsigned)nb, blk, 0, st>>>(out, a, so);
    } else {
      if (D == 0) k_permute_tiled<0, S, 32><<<(unsigned)nb, blk, 0, st>>>(out, a, so);
      if (D == 1) k_permute_tiled<1, S, 32><<<(unsigned)nb, blk, 0, st>>>(out, a, so);
      if (D == 2) k_permute_tiled<2, S, 32><<<(unsigned)nb, blk, 0, st>>>(out, a, so);
    }
    count_launch();
  } else {
    long long nb = (total + 255) / 256;
    if (nb > 148 * 64) nb = 148 * 64;
    const bool rows4 = all_unit3 && a.n[3] % 4 == 0 && total < (1LL << 31) &&
                       (!out || ((uintptr_t)out & 15) == 0);
    if (rows4) {
      long long nq = (total / 4 + 255) / 256;
      if (nq > 148 * 64) nq = 148 * 64;
      k_permute_rows4<S><<<(unsigned)nq, 256, 0, st>>>(out, a, total / 4, so);
    } else if (S || total < (1LL << 31)) {
      k_permute_naive<false, S><<<(unsigned)nb, 256, 0, st>>>(out, a, total, so);
    } else {
      k_permute_naive<true, false><<<(unsigned)nb, 256, 0, st>>>(out, a, total, so);
    }
    count_launch();
  }
}

static void perm_args(PermArgs &a, const PermSpec &spec, long long &total) {
  total = 1;
  for (int k = 0; k < 4; ++k) {
    a.n[k] = spec.n[k];
    total *= spec.n[k];
  }
  a.nterms = spec.nterms;
  a.beta = spec.beta;
  for (int t = 0; t < 4; ++t) {
    a.src[t] = t < spec.nterms ? spec.t[t].src : nullptr;
    a.alpha[t] = t < spec.nterms ? spec.t[t].alpha : 0.0;
    for (int k = 0; k < 4; ++k) a.s[t][k] = t < spec.nterms ? spec.t[t].s[k] : 0;
  }
  // merge adjacent output indices k, k+1 that every source also reads as one
  // run (s[k] = s[k+1] n[k+1]): e.g. tau[m,n,a,b] -> [a,b,(m,n)] becomes a
  // plain 2-index transpose whose inner extent o^2 fills the resort tiles
  int k = 2;
  while (k >= 0) {
    bool ok = a.n[k] > 1 && (long long)a.n[k] * a.n[k + 1] < (1LL << 31);
    for (int t = 0; t < a.nterms && ok; ++t)
      if (a.s[t][k] != a.s[t][k + 1] * a.n[k + 1]) ok = false;
    if (!ok) {
      --k;
      continue;
    }
    a.n[k + 1] *= a.n[k];
    for (int j = k; j > 0; --j) {
      a.n[j] = a.n[j - 1];
      for (int t = 0; t < 4; ++t) a.s[t][j] = a.s[t][j - 1];
    }
    a.n[0] = 1;
    for (int t = 0; t < 4; ++t) a.s[t][0] = 0;
    // the merged index (now at k + 1) may merge again with the one now at k
  }
  a.fd1 = FastDiv((unsigned)a.n[1]);
  a.fd2 = FastDiv((unsigned)a.n[2]);
  a.fd3 = FastDiv((unsigned)a.n[3]);
}

int permute(double *out, const PermSpec &spec, cudaStream_t st) {
  PermArgs a;
  long long total;
  perm_args(a, spec, total);
  if (total == 0) return ACES_OK;
  permute_launch<false>(out, a, spec, total, SplitOut(), st);
  ACES_CUDA(cudaGetLastError());
  return ACES_OK;
}

int permute_split(double *out, void *hi, void *lo, int K, int k_pad, const PermSpec &spec,
                  cudaStream_t st) {
  PermArgs a;
  long long total;
  perm_args(a, spec, total);
  if (total == 0) return ACES_OK;
  if (K < 1 || k_pad < K || total % K != 0 || total >= (1LL << 31) || spec.beta != 0.0 ||
      (!out && !hi)) {
    set_error("permute_split: %lld outputs as rows of K = %d (k_pad %d) not supported", total, K,
              k_pad);
    return ACES_ERR_ARG;
  }
  SplitOut so;
  so.hi = (__nv_bfloat16 *)hi;
  so.lo = (__nv_bfloat16 *)lo;
  so.k_pad = k_pad;
  so.fk = FastDiv((unsigned)K);
  permute_launch<true>(out, a, spec, total, so, st);
  ACES_CUDA(cudaGetLastError());
  return ACES_OK;
}

// ---------------------------------------------------------------------------
// Pair blocks of [o,o,v,v] arrays
// ---------------------------------------------------------------------------
// Work units (p, c): p a pair of occupied indices, c a chunk of kPbChunk
// consecutive (a,b) of its v*v pair block; thread t of the unit's block owns
// (a,b) = c*kPbChunk + t + kPbThreads*u for u < kPbPer, so a warp's loads are
// coalesced and each thread keeps kPbPer (twice that for two blocks) loads in
// flight without any per-element 64-bit index split.  The symmetric walks run
// p over the o(o+1)/2 pairs i <= j (p = j(j+1)/2 + i) and read the [i,j] and
// [j,i] blocks of a unit together: an element and its exchange partner
// x[j,i,a,b] (= x[i,j,b,a] for a pair-symmetric vector) meet in registers and
// every element is loaded once.
constexpr int kPbThreads = 256, kPbPer = 4, kPbChunk = kPbThreads * kPbPer;

struct PairBlocks {
  int o, v;
  long long vv;        // elements per pair block
  int nchunk;          // chunks per pair block
  long long nunits;    // pairs x chunks
  FastDiv fv;          // divisor v, for a = ab / v
};

PairBlocks pair_blocks(int o, int v, bool symmetric) {
  PairBlocks P;
  P.o = o;
  P.v = v;
  P.vv = (long long)v * v;
  P.nchunk = (int)((P.vv + kPbChunk - 1) / kPbChunk);
  const long long npair = symmetric ? (long long)o * (o + 1) / 2 : (long long)o * o;
  P.nunits = npair * P.nchunk;
  P.fv = FastDiv((unsigned)std::max(v, 1));
  return P;
}

// (i, j) with i <= j of the symmetric pair index p = j(j+1)/2 + i
__device__ __forceinline__ void pb_pair(long long p, int &i, int &j) {
  int jj = (int)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
  while ((long long)(jj + 1) * (jj + 2) / 2 <= p) ++jj;
  while ((long long)jj * (jj + 1) / 2 > p) --jj;
  j = jj;
  i = (int)(p - (long long)jj * (jj + 1) / 2);
}

// 256-thread blocks, a multiple of the SM count, at most one block per unit
inline unsigned pb_grid(long long nunits, int per_sm) {
  return (unsigned)std::max(1LL, std::min(nunits, 148LL * per_sm));
}

// tau[i,j,a,b] = t2[i,j,a,b] + c t1[i,a] t1[j,b]; units over all o^2 pairs
__global__ void __launch_bounds__(kPbThreads)
    k_tau(double *__restrict__ tau, const double *__restrict__ t2,
          const double *__restrict__ t1, double c, PairBlocks P) {
  for (long long u = blockIdx.x; u < P.nunits; u += gridDim.x) {
    const long long p = u / P.nchunk;
    const int ab0 = (int)(u - p * P.nchunk) * kPbChunk + threadIdx.x;
    const int i = (int)(p / P.o), j = (int)(p - (long long)i * P.o);
    const long long base = p * P.vv;
    double x[kPbPer];
#pragma unroll
    for (int k = 0; k < kPbPer; ++k) {
      const int ab = ab0 + k * kPbThreads;
      x[k] = ab < P.vv ? t2[base + ab] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < kPbPer; ++k) {
      const int ab = ab0 + k * kPbThreads;
      if (ab < P.vv) {
        const int a = (int)P.fv.div((unsigned)ab), b = ab - a * P.v;
        tau[base + ab] = x[k] + c * __ldg(t1 + i * P.v + a) * __ldg(t1 + j * P.v + b);
      }
    }
  }
}

void launch_tau(double *tau, const double *t2, const double *t1, double c, int o, int v,
                cudaStream_t st) {
  const PairBlocks P = pair_blocks(o, v, false);
  if (P.nunits == 0) return;
  k_tau<<<pb_grid(P.nunits, 8), kPbThreads, 0, st>>>(tau, t2, t1, c, P);
  count_launch();
}

// NEWT2 for a closed-shell pair-symmetric T2: t2n[i,j,a,b] = t2n[j,i,b,a] =
// (z2[i,j,a,b] + z2[j,i,b,a]) / 2 / (e_i + e_j - e_a - e_b).  A unit is one
// pair i <= j and one 32 x 32 (a, b) tile: the [i,j] tile (rows a) and the
// [j,i] tile (rows b) are loaded together into shared memory (8 loads in
// flight per thread); each element is divided once and both output tiles
// are written with coalesced stores (the [j,i] one through the transposed
// shared-memory read of the results).
__global__ void __launch_bounds__(256)
    k_newt(double *__restrict__ t2n, const double *__restrict__ z2, double *__restrict__ t1n,
           const double *__restrict__ z1, const double *__restrict__ eo,
           const double *__restrict__ ev, int o, int v, int tiles, long long nunits) {
  __shared__ double tz[2][32][33];   // [ij tile: a rows][ji tile: b rows]
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  // T1: z1 / (e_i - e_a)
  for (int e = blockIdx.x * 256 + threadIdx.x; e < o * v; e += gridDim.x * 256)
    t1n[e] = z1[e] / (eo[e / v] - ev[e % v]);
  const long long vv = (long long)v * v;
  const int tt = tiles * tiles;
  for (long long u = blockIdx.x; u < nunits; u += gridDim.x) {
    const long long p = u / tt;
    const int tile = (int)(u - p * tt);
    const int a0 = (tile / tiles) * 32, b0 = (tile % tiles) * 32;
    int i, j;
    pb_pair(p, i, j);
    const double *zij = z2 + ((long long)i * o + j) * vv;
    const double *zji = z2 + ((long long)j * o + i) * vv;
    double *wij = t2n + ((long long)i * o + j) * vv;
    double *wji = t2n + ((long long)j * o + i) * vv;
    double xa[4], xb[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int r = ty + 8 * k;
      const int a = a0 + r, b = b0 + tx;     // [i,j] tile element (a, b)
      xa[k] = (a < v && b < v) ? zij[(long long)a * v + b] : 0.0;
      const int bb = b0 + r, aa = a0 + tx;   // [j,i] tile element (b, a)
      xb[k] = (aa < v && bb < v) ? zji[(long long)bb * v + aa] : 0.0;
    }
    __syncthreads();  // the previous unit's tile reads are done
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      tz[0][ty + 8 * k][tx] = xa[k];
      tz[1][ty + 8 * k][tx] = xb[k];
    }
    __syncthreads();
    const double eij = eo[i] + eo[j];
    const double evb = b0 + tx < v ? ev[b0 + tx] : 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int al = ty + 8 * k, a = a0 + al, b = b0 + tx;
      if (a < v && b < v) {
        const double x = 0.5 * (tz[0][al][tx] + tz[1][tx][al]) / (eij - ev[a] - evb);
        wij[(long long)a * v + b] = x;
        tz[0][al][tx] = x;  // this thread's own position: no other thread reads it
      }
    }
    if (i == j) continue;  // block-uniform
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int bl = ty + 8 * k, b = b0 + bl, a = a0 + tx;
      if (a < v && b < v) wji[(long long)b * v + a] = tz[0][tx][bl];
    }
  }
}

void launch_newt(double *t2n, const double *z2, double *t1n, const double *z1, const double *eo,
                 const double *ev, int o, int v, cudaStream_t st) {
  const int tiles = (v + 31) / 32;
  const long long nunits = (long long)o * (o + 1) / 2 * tiles * tiles;
  // the blocks walk the units persistently: no more of them than stay
  // resident together (a second wave would start its share late)
  static int per_sm = 0;
  if (!per_sm) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_newt, 256, 0) != cudaSuccess ||
        per_sm <= 0) {
      cudaGetLastError();
      per_sm = 4;
    }
  }
  const unsigned grid = (unsigned)std::max(1LL, std::min(nunits, 148LL * per_sm));
  k_newt<<<grid, 256, 0, st>>>(t2n, z2, t1n, z1, eo, ev, o, v, tiles, nunits);
  count_launch();
}

// ---------------------------------------------------------------------------
// FP64 reductions (deterministic two-pass)
// ---------------------------------------------------------------------------
constexpr int kRedBlocks = 592;  // 4 per SM

template <int N>
__device__ void block_reduce(double (&vals)[N], double *out) {
  __shared__ double sh[N][32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int k = 0; k < N; ++k) {
    double x = vals[k];
    for (int off = 16; off; off >>= 1) x += __shfl_down_sync(0xffffffff, x, off);
    if (lane == 0) sh[k][wid] = x;
  }
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    for (int k = 0; k < N; ++k) {
      double x = lane < nw ? sh[k][lane] : 0.0;
      for (int off = 16; off; off >>= 1) x += __shfl_down_sync(0xffffffff, x, off);
      if (lane == 0) out[k] = x;
    }
  }
}

__device__ __forceinline__ double warp_sum(double x) {
  for (int off = 16; off; off >>= 1) x += __shfl_down_sync(0xffffffff, x, off);
  return x;
}

// E = sum tau[ijab] (2 V[ijab] - V[ijba]) + 2 sum f_ia t_ia, accumulated as
// s0 = sum tau V, s1 = sum tau (V[ijab] - V[ijba]) / 2, s2 = 2 sum f t1.  For
// real orbitals <ij|ba> = <ji|ab>: the exchange integral of an [i,j] element
// is the [j,i] element at the same (a, b), read in the same pair-block unit.
__global__ void __launch_bounds__(kPbThreads)
    k_energy(double *__restrict__ part, const double *__restrict__ t2,
             const double *__restrict__ t1, const double *__restrict__ V,
             const double *__restrict__ fov, PairBlocks P) {
  double s[3] = {0.0, 0.0, 0.0};
  const int n1 = P.o * P.v;
  for (int e = blockIdx.x * kPbThreads + threadIdx.x; e < n1; e += gridDim.x * kPbThreads)
    s[2] += 2.0 * fov[e] * t1[e];
  for (long long u = blockIdx.x; u < P.nunits; u += gridDim.x) {
    const long long p = u / P.nchunk;
    const int ab0 = (int)(u - p * P.nchunk) * kPbChunk + threadIdx.x;
    int i, j;
    pb_pair(p, i, j);
    const long long o1 = ((long long)i * P.o + j) * P.vv, o2 = ((long long)j * P.o + i) * P.vv;
    if (i == j) {
#pragma unroll
      for (int k = 0; k < kPbPer; ++k) {
        const int ab = ab0 + k * kPbThreads;
        if (ab < P.vv) {
          const int a = (int)P.fv.div((unsigned)ab), b = ab - a * P.v;
          const double tau = t2[o1 + ab] + __ldg(t1 + i * P.v + a) * __ldg(t1 + i * P.v + b);
          s[0] += tau * V[o1 + ab];
        }
      }
      continue;
    }
    double x1[kPbPer], x2[kPbPer], v1[kPbPer], v2[kPbPer];
#pragma unroll
    for (int k = 0; k < kPbPer; ++k) {
      const int ab = ab0 + k * kPbThreads;
      const bool in = ab < P.vv;
      x1[k] = in ? t2[o1 + ab] : 0.0;
      x2[k] = in ? t2[o2 + ab] : 0.0;
      v1[k] = in ? V[o1 + ab] : 0.0;
      v2[k] = in ? V[o2 + ab] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < kPbPer; ++k) {
      const int ab = ab0 + k * kPbThreads;
      if (ab < P.vv) {
        const int a = (int)P.fv.div((unsigned)ab), b = ab - a * P.v;
        const double tau1 = x1[k] + __ldg(t1 + i * P.v + a) * __ldg(t1 + j * P.v + b);
        const double tau2 = x2[k] + __ldg(t1 + j * P.v + a) * __ldg(t1 + i * P.v + b);
        s[0] += tau1 * v1[k] + tau2 * v2[k];
        s[1] += 0.5 * tau1 * (v1[k] - v2[k]) + 0.5 * tau2 * (v2[k] - v1[k]);
      }
    }
  }
  block_reduce<3>(s, part + 3 * blockIdx.x);
}

__global__ void k_final_sum(double *out, const double *part, int nblk, int nv) {
  // single warp per value, fixed order
  int k = blockIdx.x;
  double x = 0.0;
  for (int b = threadIdx.x; b < nblk; b += 32) x += part[(long long)b * nv + k];
  for (int off = 16; off; off >>= 1) x += __shfl_down_sync(0xffffffff, x, off);
  if (threadIdx.x == 0) out[k] = x;
}

void launch_energy(double *out3, const double *t2, const double *t1, const double *voovv,
                   const double *fov, int o, int v, double *scratch, cudaStream_t st) {
  const PairBlocks P = pair_blocks(o, v, true);
  k_energy<<<kRedBlocks, kPbThreads, 0, st>>>(scratch, t2, t1, voovv, fov, P);
  count_launch();
  k_final_sum<<<3, 32, 0, st>>>(out3, scratch, kRedBlocks, 3); count_launch();
}

// xn = x + damp (xn - x), two loads and a store per element
__global__ void k_blend(double *__restrict__ xn, const double *__restrict__ x, double damp,
                        long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    xn[i] = fma(damp, xn[i] - x[i], x[i]);
}

void launch_blend(double *xn, const double *x, double damp, long long n, cudaStream_t st) {
  long long nb = (n + 255) / 256;
  if (nb > 148 * 32) nb = 148 * 32;
  k_blend<<<(unsigned)nb, 256, 0, st>>>(xn, x, damp, n); count_launch();
}

struct HistPtrs {
  const double *p[25];
};

// signed absmax; ties resolved towards the lower index (ISAMAX)
__device__ inline void amax_merge(double &bv, long long &bi, double v, long long i) {
  if (fabs(v) > fabs(bv) || (fabs(v) == fabs(bv) && i < bi)) {
    bv = v;
    bi = i;
  }
}

// one warp; amax_merge orders candidates by (|value| descending, index
// ascending), a total order, so the merge order does not change the result
__global__ void k_absmax_final(double *out, const double *pv, const long long *pi, int nb) {
  double bv = 0.0;
  long long bi = 0x7fffffffffffffffLL;
  for (int b = threadIdx.x; b < nb; b += 32) amax_merge(bv, bi, pv[b], pi[b]);
  for (int off = 16; off; off >>= 1) {
    double ov = __shfl_down_sync(0xffffffff, bv, off);
    long long oi = __shfl_down_sync(0xffffffff, bi, off);
    amax_merge(bv, bi, ov, oi);
  }
  if (threadIdx.x == 0) out[0] = bv;
}

// block-level absmax into pv[blockIdx.x], pi[blockIdx.x]
__device__ void block_absmax(double bv, long long bi, double *pv, long long *pi) {
  __shared__ double sv[8];
  __shared__ long long si[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int off = 16; off; off >>= 1) {
    const double ov = __shfl_down_sync(0xffffffff, bv, off);
    const long long oi = __shfl_down_sync(0xffffffff, bi, off);
    amax_merge(bv, bi, ov, oi);
  }
  if (lane == 0) {
    sv[wid] = bv;
    si[wid] = bi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) amax_merge(bv, bi, sv[w], si[w]);
    pv[blockIdx.x] = bv;
    pi[blockIdx.x] = bi;
  }
}

// The absmax candidates of a pair-symmetric vector x = [T1 | T2]: every
// element (its index), and for i < j, a < b the packed same-spin amplitude
// x[i,j,a,b] - x[i,j,b,a] = x[i,j,a,b] - x[j,i,a,b] (index n1 + n2 + the
// [i,j,a,b] element's index); x1 / x2 are the [i,j] / [j,i] elements of a unit.
__device__ __forceinline__ void pb_absmax(double &bv, long long &bi, const double (&x1)[kPbPer],
                                          const double (&x2)[kPbPer], bool off, long long g1,
                                          long long g2, long long aa, int ab0,
                                          const PairBlocks &P) {
#pragma unroll
  for (int k = 0; k < kPbPer; ++k) {
    const int ab = ab0 + k * kPbThreads;
    if (ab < P.vv) {
      amax_merge(bv, bi, x1[k], g1 + ab);
      if (off) {
        amax_merge(bv, bi, x2[k], g2 + ab);
        const int a = (int)P.fv.div((unsigned)ab), b = ab - a * P.v;
        if (a < b) amax_merge(bv, bi, x1[k] - x2[k], aa + g1 + ab);
      }
    }
  }
}

// One pass over the new DIIS error vector e = xnew - xold: writes e, its
// signed absmax over T1, T2(AB) and packed T2(AA), and its dots with the nh
// history error vectors, where the dot of two pair-symmetric vectors over
// T1, T2(AB) and packed T2(AA) (i<j, a<b) is
//   sum x y + sum_{i<j} sum_ab x_ijab (y_ijab - y_jiab)
// (history slot `self` is e itself, taken from registers).  Per unit and
// history slot a warp sums its lanes' products and lane 0 adds the sum to the
// warp's shared slot: a fixed order, so the dots are deterministic.
__global__ void __launch_bounds__(kPbThreads)
    k_diff_stats(double *__restrict__ e, const double *__restrict__ xnew,
                 const double *__restrict__ xold, HistPtrs h, int nh, int self, PairBlocks P,
                 double *__restrict__ part, double *__restrict__ pv, long long *__restrict__ pi) {
  __shared__ double sh[25][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
    for (int k = 0; k < 25; ++k) sh[k][wid] = 0.0;
  const long long n1 = (long long)P.o * P.v, n2 = (long long)P.o * P.o * P.vv;
  double bv = 0.0;
  long long bi = 0x7fffffffffffffffLL;
  // T1
  for (int k = 0; k < nh; ++k) {
    double acc = 0.0;
    for (long long idx = blockIdx.x * kPbThreads + threadIdx.x; idx < n1;
         idx += (long long)gridDim.x * kPbThreads) {
      const double x = xnew[idx] - xold[idx];
      if (k == 0) {
        e[idx] = x;
        amax_merge(bv, bi, x, idx);
      }
      acc += x * (k == self ? x : h.p[k][idx]);
    }
    acc = warp_sum(acc);
    if (lane == 0) sh[k][wid] += acc;
  }
  // T2, by pair-block units
  for (long long u = blockIdx.x; u < P.nunits; u += gridDim.x) {
    const long long p = u / P.nchunk;
    const int ab0 = (int)(u - p * P.nchunk) * kPbChunk + threadIdx.x;
    int i, j;
    pb_pair(p, i, j);
    const bool off = i != j;
    const long long g1 = n1 + ((long long)i * P.o + j) * P.vv;
    const long long g2 = n1 + ((long long)j * P.o + i) * P.vv;
    double x1[kPbPer], x2[kPbPer];
#pragma unroll
    for (int k = 0; k < kPbPer; ++k) {
      const int ab = ab0 + k * kPbThreads;
      const bool in = ab < P.vv;
      x1[k] = in ? xnew[g1 + ab] - xold[g1 + ab] : 0.0;
      x2[k] = in && off ? xnew[g2 + ab] - xold[g2 + ab] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < kPbPer; ++k) {
      const int ab = ab0 + k * kPbThreads;
      if (ab < P.vv) {
        e[g1 + ab] = x1[k];
        if (off) e[g2 + ab] = x2[k];
      }
    }
    pb_absmax(bv, bi, x1, x2, off, g1, g2, n2, ab0, P);
    for (int k = 0; k < nh; ++k) {
      double acc = 0.0;
      if (k == self) {
#pragma unroll
        for (int q = 0; q < kPbPer; ++q)
          acc += x1[q] * x1[q] + (off ? x1[q] * (x1[q] - x2[q]) + x2[q] * x2[q] : 0.0);
      } else {
        const double *y = h.p[k];
        double y1[kPbPer], y2[kPbPer];
#pragma unroll
        for (int q = 0; q < kPbPer; ++q) {
          const int ab = ab0 + q * kPbThreads;
          const bool in = ab < P.vv;
          y1[q] = in ? y[g1 + ab] : 0.0;
          y2[q] = in && off ? y[g2 + ab] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < kPbPer; ++q)
          acc += x1[q] * y1[q] + (off ? x1[q] * (y1[q] - y2[q]) + x2[q] * y2[q] : 0.0);
      }
      acc = warp_sum(acc);
      if (lane == 0) sh[k][wid] += acc;
    }
  }
  __syncthreads();
  if (threadIdx.x < nh) {
    double x = 0.0;
    for (int w = 0; w < kPbThreads / 32; ++w) x += sh[threadIdx.x][w];
    part[(long long)blockIdx.x * 25 + threadIdx.x] = x;
  }
  block_absmax(bv, bi, pv, pi);
}

int launch_diff_stats(double *e, const double *xnew, const double *xold,
                      const double *const *hist, int nh, int self, int o, int v,
                      double *scratch, double *absmax_out, double *dots_out, cudaStream_t st) {
  if (nh < 1 || nh > 25 || self < 0 || self >= nh) return ACES_ERR_ARG;
  HistPtrs h;
  for (int k = 0; k < 25; ++k) h.p[k] = k < nh ? hist[k] : nullptr;
  double *part = scratch;                   // [kRedBlocks][25]
  double *pv = scratch + kRedBlocks * 25;   // [kRedBlocks]
  long long *pi = (long long *)(scratch + kRedBlocks * 26);
  const PairBlocks P = pair_blocks(o, v, true);
  k_diff_stats<<<kRedBlocks, kPbThreads, 0, st>>>(e, xnew, xold, h, nh, self, P, part, pv, pi);
  count_launch();
  k_absmax_final<<<1, 32, 0, st>>>(absmax_out, pv, pi, kRedBlocks);
  count_launch();
  k_final_sum<<<nh, 32, 0, st>>>(dots_out, part, kRedBlocks, 25);
  count_launch();
  ACES_CUDA(cudaGetLastError());
  return ACES_OK;
}

// out = sum_k c[k] p_k over a pair-symmetric [T1 | T2] (the DIIS residual of
// the stored error vectors) with its signed absmax (as k_diff_stats) in the
// same pass; the sums run over k in order, element by element.
__global__ void __launch_bounds__(kPbThreads)
    k_lincomb_absmax(double *__restrict__ out, const double *__restrict__ c, HistPtrs hp, int n,
                     PairBlocks P, double *__restrict__ pv, long long *__restrict__ pi) {
  __shared__ double cs[25];
  if (threadIdx.x < n) cs[threadIdx.x] = c[threadIdx.x];
  __syncthreads();
  const long long n1 = (long long)P.o * P.v, n2 = (long long)P.o * P.o * P.vv;
  double bv = 0.0;
  long long bi = 0x7fffffffffffffffLL;
  for (long long idx = blockIdx.x * kPbThreads + threadIdx.x; idx < n1;
       idx += (long long)gridDim.x * kPbThreads) {
    double acc = 0.0;
    for (int k = 0; k < n; ++k) acc += cs[k] * hp.p[k][idx];
    out[idx] = acc;
    amax_merge(bv, bi, acc, idx);
  }
  for (long long u = blockIdx.x; u < P.nunits; u += gridDim.x) {
    const long long p = u / P.nchunk;
    const int ab0 = (int)(u - p * P.nchunk) * kPbChunk + threadIdx.x;
    int i, j;
    pb_pair(p, i, j);
    const bool off = i != j;
    const long long g1 = n1 + ((long long)i * P.o + j) * P.vv;
    const long long g2 = n1 + ((long long)j * P.o + i) * P.vv;
    double x1[kPbPer], x2[kPbPer];
#pragma unroll
    for (int q = 0; q < kPbPer; ++q) x1[q] = x2[q] = 0.0;
    for (int k = 0; k < n; ++k) {
      // all loads of a history vector issued before its products are added
      const double *y = hp.p[k];
      const double ck = cs[k];
      double y1[kPbPer], y2[kPbPer];
#pragma unroll
      for (int q = 0; q < kPbPer; ++q) {
        const int ab = ab0 + q * kPbThreads;
        y1[q] = ab < P.vv ? y[g1 + ab] : 0.0;
        y2[q] = ab < P.vv && off ? y[g2 + ab] : 0.0;
      }
#pragma unroll
      for (int q = 0; q < kPbPer; ++q) {
        x1[q] += ck * y1[q];
        x2[q] += ck * y2[q];
      }
    }
#pragma unroll
    for (int q = 0; q < kPbPer; ++q) {
      const int ab = ab0 + q * kPbThreads;
      if (ab < P.vv) {
        out[g1 + ab] = x1[q];
        if (off) out[g2 + ab] = x2[q];
      }
    }
    pb_absmax(bv, bi, x1, x2, off, g1, g2, n2, ab0, P);
  }
  block_absmax(bv, bi, pv, pi);
}

void launch_lincomb_absmax(double *out, const double *c, const double *const *p, int n, int o,
                           int v, double *scratch, double *absmax_out, cudaStream_t st) {
  HistPtrs a;
  for (int k = 0; k < 25; ++k) a.p[k] = k < n ? p[k] : nullptr;
  double *pv = scratch;
  long long *pi = (long long *)(scratch + kRedBlocks);
  const PairBlocks P = pair_blocks(o, v, true);
  k_lincomb_absmax<<<kRedBlocks, kPbThreads, 0, st>>>(out, c, a, n, P, pv, pi);
  count_launch();
  k_absmax_final<<<1, 32, 0, st>>>(absmax_out, pv, pi, kRedBlocks);
  count_launch();
}

// Bordered DIIS system [[0,-1..],[-1,B]] (lam,c) = (-1,0,..) by LU with
// partial pivoting (the pivot order of LAPACK dgetf2, libr/dodiis.F:46).
__global__ void k_diis_solve(double *coef, int *status, const double *B, int n) {
  if (threadIdx.x != 0) return;
  double A[26][26];
  double rhs[26];
  int N = n + 1;
  for (int i = 0; i < N; ++i) {
    rhs[i] = i == 0 ? -1.0 : 0.0;
    for (int j = 0; j < N; ++j) {
      if (i == 0 && j == 0) A[i][j] = 0.0;
      else if (i == 0 || j == 0) A[i][j] = -1.0;
      else A[i][j] = B[(i - 1) * 25 + (j - 1)];
    }
  }
  int st = 0;
  for (int k = 0; k < N; ++k) {
    int p = k;
    double m = fabs(A[k][k]);
    for (int i = k + 1; i < N; ++i)
      if (fabs(A[i][k]) > m) { m = fabs(A[i][k]); p = i; }
    if (m == 0.0) { st = 1; break; }
    if (p != k) {
      for (int j = 0; j < N; ++j) { double t = A[k][j]; A[k][j] = A[p][j]; A[p][j] = t; }
      double t = rhs[k]; rhs[k] = rhs[p]; rhs[p] = t;
    }
    double inv = 1.0 / A[k][k];
    for (int i = k + 1; i < N; ++i) {
      double l = A[i][k] * inv;
      A[i][k] = l;
      for (int j = k + 1; j < N; ++j) A[i][j] -= l * A[k][j];
      rhs[i] -= l * rhs[k];
    }
  }
  if (!st) {
    for (int i = N - 1; i >= 0; --i) {
      double x = rhs[i];
      for (int j = i + 1; j < N; ++j) x -= A[i][j] * rhs[j];
      rhs[i] = x / A[i][i];
    }
    for (int i = 0; i < n; ++i) coef[i] = rhs[i + 1];
  }
  status[0] = st;
}

void launch_diis_solve(double *coef_out, int *status_out, const double *B, int n, cudaStream_t st) {
  k_diis_solve<<<1, 32, 0, st>>>(coef_out, status_out, B, n); count_launch();
}

__global__ void k_lincomb(double *__restrict__ out, const double *__restrict__ base,
                          const double *__restrict__ c, HistPtrs p, int n, long long len) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x) {
    double acc = base ? base[i] : 0.0;
    for (int k = 0; k < n; ++k) acc += c[k] * p.p[k][i];
    out[i] = acc;
  }
}

void launch_lincomb(double *out, const double *base, const double *c, const double *const *p,
                    int n, long long len, cudaStream_t st) {
  HistPtrs a;
  for (int k = 0; k < 25; ++k) a.p[k] = k < n ? p[k] : nullptr;
  long long nb = (len + 255) / 256;
  if (nb > 148 * 32) nb = 148 * 32;
  k_lincomb<<<(unsigned)nb, 256, 0, st>>>(out, base, c, a, n, len); count_launch();
}

// ---------------------------------------------------------------------------
// DPD list <-> dense
// ---------------------------------------------------------------------------
__global__ void k_gather(double *__restrict__ dense, DpdMap m, long long total) {
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    long long r = idx;
    int s = r % m.ns; r /= m.ns;
    int q2 = r % m.nr; r /= m.nr;
    int q = r % m.nq;
    int p = (int)(r / m.nq);
    int hpq = m.irr_p[p] ^ m.irr_q[q];
    int hrs = m.irr_r[q2] ^ m.irr_s[s];
    double val = 0.0;
    if (hpq == hrs) {
      int ri = m.rowidx[p * m.nq + q], ci = m.colidx[q2 * m.ns + s];
      if (ri >= 0 && ci >= 0) {
        int a = m.rowsgn[p * m.nq + q], b = m.colsgn[q2 * m.ns + s];
        double sg = (double)(a == 2 ? 1 : a) * (double)(b == 2 ? 1 : b);
        val = sg * m.base[hrs][(long long)ci * m.nrows[hrs] + ri];
      }
    }
    dense[idx] = val;
  }
}

__global__ void k_scatter(const double *__restrict__ dense, DpdMap m, long long total) {
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    long long r = idx;
    int s = r % m.ns; r /= m.ns;
    int q2 = r % m.nr; r /= m.nr;
    int q = r % m.nq;
    int p = (int)(r / m.nq);
    int hpq = m.irr_p[p] ^ m.irr_q[q];
    int hrs = m.irr_r[q2] ^ m.irr_s[s];
    if (hpq != hrs) continue;
    int ri = m.rowidx[p * m.nq + q], ci = m.colidx[q2 * m.ns + s];
    // write only the canonical (positive-sign) representative of packed pairs
    if (ri < 0 || ci < 0) continue;
    if (m.rowsgn[p * m.nq + q] != 1 || m.colsgn[q2 * m.ns + s] != 1) continue;
    m.base[hrs][(long long)ci * m.nrows[hrs] + ri] = dense[idx];
  }
}

// The same scatter from X[r][p][s][q] (the row-major product of the
// integral producer, m = (r,p), n = (s,q)), read in its own order so the loads
// coalesce; every pair type involved stores all of its pairs (FULL).
__global__ void k_scatter_rpsq(const double *__restrict__ X, DpdMap m, long long total) {
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    long long t = idx;
    const int q = (int)(t % m.nq); t /= m.nq;
    const int s = (int)(t % m.ns); t /= m.ns;
    const int p = (int)(t % m.np);
    const int r = (int)(t / m.np);
    const int hpq = m.irr_p[p] ^ m.irr_q[q];
    const int hrs = m.irr_r[r] ^ m.irr_s[s];
    if (hpq != hrs) continue;
    const int ri = m.rowidx[p * m.nq + q], ci = m.colidx[r * m.ns + s];
    if (ri < 0 || ci < 0) continue;
    m.base[hrs][(long long)ci * m.nrows[hrs] + ri] = X[idx];
  }
}

void launch_scatter_rpsq(const double *X, const DpdMap &m, cudaStream_t st) {
  long long total = (long long)m.np * m.nq * m.nr * m.ns;
  long long nb = (total + 255) / 256;
  if (nb > 148 * 32) nb = 148 * 32;
  if (nb < 1) nb = 1;
  k_scatter_rpsq<<<(unsigned)nb, 256, 0, st>>>(X, m, total); count_launch();
}

void launch_gather(double *dense, const DpdMap &m, cudaStream_t st) {
  long long total = (long long)m.np * m.nq * m.nr * m.ns;
  long long nb = (total + 255) / 256;
  if (nb > 148 * 32) nb = 148 * 32;
  if (nb < 1) nb = 1;
  k_gather<<<(unsigned)nb, 256, 0, st>>>(dense, m, total); count_launch();
}

void launch_scatter(const double *dense, const DpdMap &m, cudaStream_t st) {
  long long total = (long long)m.np * m.nq * m.nr * m.ns;
  long long nb = (total + 255) / 256;
  if (nb > 148 * 32) nb = 148 * 32;
  if (nb < 1) nb = 1;
  k_scatter<<<(unsigned)nb, 256, 0, st>>>(dense, m, total); count_launch();
}

// ---------------------------------------------------------------------------
// Packed particle-particle ladder
// ---------------------------------------------------------------------------
// U+[p(a,b)][p(c,d)] = (V[ab,cd] + V[ab,dc]) / 2 (c < d), V[ab,cc];
// U-[m(a,b)][m(c,d)] = (V[ab,cd] - V[ab,dc]) / 2, p(c,d) = d(d+1)/2 + c,
// m(c,d) = d(d-1)/2 + c.  One block per (row a <= b, 32 x 32 tile pair of
// (c, d) with the c tile <= the d tile): the [c][d] and [d][c] tiles of the
// row's v x v block are read coalesced, the second through a shared-memory
// transpose, and the packed outputs (consecutive c for one d) coalesce.
__global__ void __launch_bounds__(256)
    k_ladder_pack_v(double *__restrict__ Up, double *__restrict__ Um,
                    const double *__restrict__ V, const int *__restrict__ pairs, int v,
                    int ntile) {
  __shared__ double t1[32][33];  // [c][d]
  __shared__ double t2[32][33];  // [c][d] = V[ab][d][c]
  const int np = v * (v + 1) / 2, nm = v * (v - 1) / 2;
  const int npairs_t = ntile * (ntile + 1) / 2;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const size_t vv = (size_t)v * v;
  for (long long blk = blockIdx.x; blk < (long long)np * npairs_t; blk += gridDim.x) {
    const int r = (int)(blk / npairs_t);
    int tp = (int)(blk - (long long)r * npairs_t);
    // tile pair tp -> (tc <= td)
    int td = 0;
    while ((td + 1) * (td + 2) / 2 <= tp) ++td;
    const int tc = tp - td * (td + 1) / 2;
    const int a = pairs[2 * r], b = pairs[2 * r + 1];
    const double *row = V + ((size_t)a * v + b) * vv;
    const int c0 = tc * 32, d0 = td * 32;
    __syncthreads();  // the previous tile's reads of t1/t2 are done
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int cl = ty + 8 * k;
      const int c = c0 + cl, d = d0 + tx;
      t1[cl][tx] = (c < v && d < v) ? row[(size_t)c * v + d] : 0.0;  // along d
      const int dl = ty + 8 * k;
      const int dd = d0 + dl, cc = c0 + tx;
      t2[tx][dl] = (cc < v && dd < v) ? row[(size_t)dd * v + cc] : 0.0;  // along c
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int dl = ty + 8 * k, cl = tx;
      const int c = c0 + cl, d = d0 + dl;
      if (c >= v || d >= v || c > d) continue;
      const double x = t1[cl][dl], y = t2[cl][dl];
      if (c == d) {
        Up[(size_t)r * np + (size_t)d * (d + 1) / 2 + c] = x;
      } else {
        Up[(size_t)r * np + (size_t)d * (d + 1) / 2 + c] = 0.5 * (x + y);
        if (a < b) Um[(size_t)(b * (b - 1) / 2 + a) * nm + (size_t)d * (d - 1) / 2 + c] =
            0.5 * (x - y);
      }
    }
  }
}

void launch_ladder_pack_v(double *Up, double *Um, const double *V, const int *pairs, int v,
                          cudaStream_t st) {
  const int ntile = (v + 31) / 32;
  const long long blocks = (long long)(v * (v + 1) / 2) * (ntile * (ntile + 1) / 2);
  k_ladder_pack_v<<<(unsigned)std::min<long long>(blocks, 148 * 64), 256, 0, st>>>(
      Up, Um, V, pairs, v, ntile);
  count_launch();
}

// tau+[ij][p(c,d)] = tau[ij][cd] + tau[ij][dc] (c < d), tau[ij][cc];
// tau-[ij][m(c,d)] = tau[ij][cd] - tau[ij][dc]
// tau+[ij][p(c,d)] = tau[ij][c][d] + tau[ij][d][c] (c < d), tau[ij][c][c] (c = d) and
// tau-[ij][m(c,d)] = tau[ij][c][d] - tau[ij][d][c] (c < d), with the packed
// indices p(c,d) = d(d+1)/2 + c and m(c,d) = d(d-1)/2 + c.  A block takes one
// ij and one 32 x 32 tile pair (c tile <= d tile): the [d][c] tile is read
// with lanes along c (the packed outputs' order), the [c][d] tile with lanes
// along d and transposed through shared memory, so every load and store is
// coalesced.  S: tau+- go straight to the BF16 planes of the ladder's B
// operands (rows ij, k_pad apart) instead of FP64 arrays.
template <bool S>
__global__ void __launch_bounds__(256)
    k_ladder_pack_tau(double *__restrict__ tp, double *__restrict__ tm,
                      const double *__restrict__ tau, int v, int noo, LadderPlanes pl) {
  __shared__ double X[32][33];  // [c local][d local] of tau[ij][c][d]
  const int np = v * (v + 1) / 2, nm = v * (v - 1) / 2;
  const size_t vv = (size_t)v * v;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  // tile pair index -> (ct <= dt), dt-major
  int dt = (int)((sqrtf(8.0f * blockIdx.x + 1.0f) - 1.0f) * 0.5f);
  while (dt * (dt + 1) / 2 > (int)blockIdx.x) --dt;
  while ((dt + 1) * (dt + 2) / 2 <= (int)blockIdx.x) ++dt;
  const int ct = blockIdx.x - dt * (dt + 1) / 2;
  const int c0 = ct * 32, d0 = dt * 32;
  for (int ij = blockIdx.y; ij < noo; ij += gridDim.y) {
    const double *t = tau + (size_t)ij * vv;
    double y[4];  // tau[d][c], lanes along c
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int cl = ty + 8 * k, c = c0 + cl, d = d0 + tx;
      X[cl][tx] = (c < v && d < v) ? t[(size_t)c * v + d] : 0.0;
      const int dd = d0 + ty + 8 * k, cc = c0 + tx;
      y[k] = (dd < v && cc < v) ? t[(size_t)dd * v + cc] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int dl = ty + 8 * k, d = d0 + dl, c = c0 + tx;
      if (c < v && d < v && c <= d) {
        const double cd = X[tx][dl], dc = y[k];
        const double plus = c == d ? cd : cd + dc;
        const size_t ip = (size_t)ij * np + (size_t)d * (d + 1) / 2 + c;
        if (!S) {
          tp[ip] = plus;
          if (c < d) tm[(size_t)ij * nm + (size_t)d * (d - 1) / 2 + c] = cd - dc;
        } else {
          __nv_bfloat16 h, l;
          split_bf16(plus, h, l);
          const size_t ap = (size_t)ij * pl.kp_p + (size_t)d * (d + 1) / 2 + c;
          pl.hi_p[ap] = h;
          pl.lo_p[ap] = l;
          if (c < d) {
            split_bf16(cd - dc, h, l);
            const size_t am = (size_t)ij * pl.kp_m + (size_t)d * (d - 1) / 2 + c;
            pl.hi_m[am] = h;
            pl.lo_m[am] = l;
          }
        }
      }
    }
    __syncthreads();  // X is reused by the next ij
  }
}

void launch_ladder_pack_tau(double *tp, double *tm, const double *tau, int v, int noo,
                            cudaStream_t st, const LadderPlanes *planes) {
  const int tiles = (v + 31) / 32;
  dim3 grid((unsigned)(tiles * (tiles + 1) / 2), (unsigned)std::min(noo, 65535));
  if (planes)
    k_ladder_pack_tau<true><<<grid, 256, 0, st>>>(tp, tm, tau, v, noo, *planes);
  else
    k_ladder_pack_tau<false><<<grid, 256, 0, st>>>(tp, tm, tau, v, noo, LadderPlanes());
  count_launch();
}

// Z2[ij][a][b] += S[ij][p] + A[ij][m] (a < b), S - A (a > b), S[ij][p(a,a)] (a = b).
// A block takes one ij and one 32 x 32 tile pair (a tile <= b tile): S and A
// are read with lanes along a (their packed order), Z2[b][a] is updated with
// lanes along a and Z2[a][b] through a shared-memory transpose with lanes
// along b, so every access is coalesced.
__global__ void __launch_bounds__(256)
    k_ladder_unpack(double *__restrict__ Z2, const double *__restrict__ S,
                    const double *__restrict__ A, int v, int noo) {
  __shared__ double P[32][33];  // S + A at [b local][a local]
  const int np = v * (v + 1) / 2, nm = v * (v - 1) / 2;
  const size_t vv = (size_t)v * v;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  int bt = (int)((sqrtf(8.0f * blockIdx.x + 1.0f) - 1.0f) * 0.5f);
  while (bt * (bt + 1) / 2 > (int)blockIdx.x) --bt;
  while ((bt + 1) * (bt + 2) / 2 <= (int)blockIdx.x) ++bt;
  const int at = blockIdx.x - bt * (bt + 1) / 2;
  const int a0 = at * 32, b0 = bt * 32;
  for (int ij = blockIdx.y; ij < noo; ij += gridDim.y) {
    double *z = Z2 + (size_t)ij * vv;
    const double *s = S + (size_t)ij * np, *an = A + (size_t)ij * nm;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int bl = ty + 8 * k, b = b0 + bl, a = a0 + tx;
      double plus = 0.0;
      if (a < v && b < v && a <= b) {
        const double sv = s[(size_t)b * (b + 1) / 2 + a];
        if (a == b) {
          z[(size_t)a * v + a] += sv;
        } else {
          const double av = an[(size_t)b * (b - 1) / 2 + a];
          z[(size_t)b * v + a] += sv - av;  // Z[b][a], lanes along a
          plus = sv + av;
        }
      }
      P[bl][tx] = plus;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int al = ty + 8 * k, a = a0 + al, b = b0 + tx;
      if (a < v && b < v && a < b) z[(size_t)a * v + b] += P[tx][al];  // Z[a][b], lanes along b
    }
    __syncthreads();
  }
}

void launch_ladder_unpack(double *Z2, const double *S, const double *A, int v, int noo,
                          cudaStream_t st) {
  const int tiles = (v + 31) / 32;
  dim3 grid((unsigned)(tiles * (tiles + 1) / 2), (unsigned)std::min(noo, 65535));
  k_ladder_unpack<<<grid, 256, 0, st>>>(Z2, S, A, v, noo);
  count_launch();
}

// ---- irrep-blocked packed ladder ----------------------------------------------
// block g of a flat index over blocks with sizes given by a prefix array
__device__ __forceinline__ int find_block(const long long *pref, int nb, long long e) {
  int g = 0;
  while (g + 1 < nb && e >= pref[g + 1]) ++g;
  return g;
}

__global__ void k_ladder_pack_v_blk(double *__restrict__ Up, double *__restrict__ Um,
                                    const double *__restrict__ V, LadderBlocks L) {
  const size_t v = L.v, vv = v * v;
  const long long nup = L.offUp[L.nirrep], total = nup + L.offUm[L.nirrep];
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    if (e < nup) {
      const int g = find_block(L.offUp, L.nirrep, e);
      const long long r = e - L.offUp[g];
      const int n = L.nP[g], pl = (int)(r / n), ql = (int)(r - (long long)pl * n);
      const int a = L.pp[2 * (L.offP[g] + pl)], b = L.pp[2 * (L.offP[g] + pl) + 1];
      const int c = L.pp[2 * (L.offP[g] + ql)], d = L.pp[2 * (L.offP[g] + ql) + 1];
      const double *row = V + ((size_t)a * v + b) * vv;
      Up[e] = c == d ? row[(size_t)c * v + c] : 0.5 * (row[(size_t)c * v + d] + row[(size_t)d * v + c]);
    } else {
      const long long em = e - nup;
      const int g = find_block(L.offUm, L.nirrep, em);
      const long long r = em - L.offUm[g];
      const int n = L.nM[g], pl = (int)(r / n), ql = (int)(r - (long long)pl * n);
      const int a = L.mm[2 * (L.offM[g] + pl)], b = L.mm[2 * (L.offM[g] + pl) + 1];
      const int c = L.mm[2 * (L.offM[g] + ql)], d = L.mm[2 * (L.offM[g] + ql) + 1];
      const double *row = V + ((size_t)a * v + b) * vv;
      Um[em] = 0.5 * (row[(size_t)c * v + d] - row[(size_t)d * v + c]);
    }
  }
}

void launch_ladder_pack_v_blk(double *Up, double *Um, const double *V, const LadderBlocks &L,
                              cudaStream_t st) {
  const long long total = L.offUp[L.nirrep] + L.offUm[L.nirrep];
  if (total == 0) return;
  const long long nb = std::min<long long>((total + 255) / 256, 148 * 32);
  k_ladder_pack_v_blk<<<(unsigned)nb, 256, 0, st>>>(Up, Um, V, L);
  count_launch();
}

__global__ void k_ladder_pack_tau_blk(double *__restrict__ tp, double *__restrict__ tm,
                                      const double *__restrict__ tau, LadderBlocks L) {
  const size_t v = L.v, vv = v * v;
  const long long ntp = L.offTp[L.nirrep], total = ntp + L.offTm[L.nirrep];
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const bool plus = e < ntp;
    const long long ee = plus ? e : e - ntp;
    const int g = find_block(plus ? L.offTp : L.offTm, L.nirrep, ee);
    const long long r = ee - (plus ? L.offTp[g] : L.offTm[g]);
    const int n = plus ? L.nP[g] : L.nM[g];
    const int rl = (int)(r / n), ql = (int)(r - (long long)rl * n);
    const int ij = L.ijs[L.offIJ[g ^ L.hs] + rl];
    const int *pl = plus ? L.pp + 2 * (L.offP[g] + ql) : L.mm + 2 * (L.offM[g] + ql);
    const int c = pl[0], d = pl[1];
    const double *t = tau + (size_t)ij * vv;
    if (plus)
      tp[e] = c == d ? t[(size_t)c * v + c] : t[(size_t)c * v + d] + t[(size_t)d * v + c];
    else
      tm[ee] = t[(size_t)c * v + d] - t[(size_t)d * v + c];
  }
}

void launch_ladder_pack_tau_blk(double *tp, double *tm, const double *tau, const LadderBlocks &L,
                                cudaStream_t st) {
  const long long total = L.offTp[L.nirrep] + L.offTm[L.nirrep];
  if (total == 0) return;
  const long long nb = std::min<long long>((total + 255) / 256, 148 * 32);
  k_ladder_pack_tau_blk<<<(unsigned)nb, 256, 0, st>>>(tp, tm, tau, L);
  count_launch();
}

// Z2[ij][a][b] += S + A / S - A / S over the elements whose pair irreps
// satisfy irrep(ab) ^ irrep(ij) == hs; S, A: block g = irrep(ab), column
// ij's local index within the occupied pairs of irrep g ^ hs
__global__ void k_ladder_unpack_blk(double *__restrict__ Z2, const double *__restrict__ S,
                                    const double *__restrict__ A, LadderBlocks L) {
  const long long v = L.v, vv = v * v, total = (long long)L.o * L.o * vv;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int ij = (int)(e / vv);
    const int ab = (int)(e - (long long)ij * vv);
    const int a = ab / (int)v, b = ab - a * (int)v;
    const int i = ij / L.o, j = ij - i * L.o;
    const int g = L.irr_v[a] ^ L.irr_v[b];
    if ((g ^ L.irr_o[i] ^ L.irr_o[j]) != L.hs) continue;
    const long long rl = L.ijl[ij];
    const double *s = S + L.offTp[g] + rl * L.nP[g];
    const double *an = A + L.offTm[g] + rl * L.nM[g];
    double x;
    if (a == b) {
      x = s[L.pidx[ab]];
    } else if (a < b) {
      x = s[L.pidx[ab]] + an[L.midx[ab]];
    } else {
      const int ba = b * (int)v + a;
      x = s[L.pidx[ba]] - an[L.midx[ba]];
    }
    Z2[e] += x;
  }
}

void launch_ladder_unpack_blk(double *Z2, const double *S, const double *A,
                              const LadderBlocks &L, cudaStream_t st) {
  const long long total = (long long)L.o * L.o * L.v * L.v;
  const long long nb = std::min<long long>((total + 255) / 256, 148 * 32);
  k_ladder_unpack_blk<<<(unsigned)std::max(1LL, nb), 256, 0, st>>>(Z2, S, A, L);
  count_launch();
}

}  // namespace acesb200
