// triples.cu -- the (T) correction (trp/trps.F -> trp/trps2.F, trp/d1t2new.F,
// librt3/rmd314.f, trp/e4tijk.F, trp/t1t32n.f) on the device.
//
// For every occupied triplet i >= j >= k the connected triples
//   W_ijk^abc = sum over the 6 simultaneous permutations of (ia)(jb)(kc) of
//     X_ijk^abc = sum_d t(ij,ad) (bd|ck) - sum_l t(il,ab) (ck|jl)
// are built in one v^3 FP64 buffer by three tensor-core launches (the 12
// contractions grouped by output orientation, four K segments each) whose
// outputs land in place through coalesced two-level views.  The energy kernel
// then sums, for the distinct permutations of (i,j,k) and all orderings of
// every virtual set {a>=b>=c}, the closed-shell expression
//   E[4]T  = 1/3 sum (4W_abc + W_bca + W_cab)(W_abc - W_cba)/D_ijk^abc
//   E[5]ST = 1/3 sum (4W_abc + W_bca + W_cab)(V_abc - V_cba)/D_ijk^abc,
//   V - W = t_i^a (jb|kc) + t_j^b (ia|kc) + t_k^c (ia|jb),
// reading every W element once per triplet.  Partial sums are kept per
// (triplet, block) and reduced in a fixed order: the FP64 energy sum is
// deterministic.
#include <algorithm>
#include <cmath>
#include <functional>
#include <vector>

#include "engine.cuh"

namespace acesb200 {

namespace {
// The six orderings s of a virtual set x = (x0, x1, x2): ordering s reads
// W at (x[kOrd[s][0]], x[kOrd[s][1]], x[kOrd[s][2]]).
constexpr int kOrd[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

constexpr int ord_index(int a, int b, int c) {
  for (int s = 0; s < 6; ++s)
    if (kOrd[s][0] == a && kOrd[s][1] == b && kOrd[s][2] == c) return s;
  return -1;
}

// kT.v[q][p][m]: for the triplet permutation p and the set ordering q, the
// ordering of the set that supplies W_abc, W_bca, W_cab and W_cba (m = 0..3)
// of the closed-shell energy expression.  Built at compile time so the
// energy kernel indexes its six W values with constants (registers).
struct TripleTable {
  int v[6][6][4];
};
constexpr TripleTable make_triple_table() {
  TripleTable t{};
  const int args[4][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  int S[6][4] = {};
  int comp[6][6] = {};
  for (int p = 0; p < 6; ++p)
    for (int m = 0; m < 4; ++m) {
      int pos[3] = {0, 0, 0};
      for (int r = 0; r < 3; ++r) pos[kOrd[p][r]] = args[m][r];
      S[p][m] = ord_index(pos[0], pos[1], pos[2]);
    }
  for (int q = 0; q < 6; ++q)
    for (int s = 0; s < 6; ++s)
      comp[q][s] = ord_index(kOrd[q][kOrd[s][0]], kOrd[q][kOrd[s][1]], kOrd[q][kOrd[s][2]]);
  for (int q = 0; q < 6; ++q)
    for (int p = 0; p < 6; ++p)
      for (int m = 0; m < 4; ++m) t.v[q][p][m] = comp[q][S[p][m]];
  return t;
}
constexpr TripleTable kT = make_triple_table();

// the table entries as template constants (usable in device code)
template <int Q, int P, int M>
struct TT {
  static constexpr int value = kT.v[Q][P][M];
};
template <int Q, int P>
__device__ __forceinline__ void accum_orders(const double (&u)[6], const double (&vd)[6],
                                             double &g4, double &g5) {
  constexpr int s0 = TT<Q, P, 0>::value, s1 = TT<Q, P, 1>::value, s2 = TT<Q, P, 2>::value,
                s3 = TT<Q, P, 3>::value;
  const double Z = 4.0 * u[s0] + u[s1] + u[s2];
  g4 += Z * (u[s0] - u[s3]);
  g5 += Z * (vd[s0] - vd[s3]);
  if constexpr (P < 5) accum_orders<Q, P + 1>(u, vd, g4, g5);
}
template <int Q>
__device__ __forceinline__ void accum_sets(const bool (&use)[6], const double (&u)[6],
                                           const double (&vd)[6], double &g4, double &g5) {
  if (use[Q]) accum_orders<Q, 0>(u, vd, g4, g5);
  if constexpr (Q < 5) accum_sets<Q + 1>(use, u, vd, g4, g5);
}

// For a set of three distinct virtuals every ordering q is used, and the
// energy terms above form a fixed bilinear form in the six W values:
//   g4 = sum_{q,p} (4 u_s0 + u_s1 + u_s2)(u_s0 - u_s3) = u^T M u,
//   g5 = sum_{q,p} (4 u_s0 + u_s1 + u_s2)(vd_s0 - vd_s3) = u^T M vd,
// with integer M[a][b] = sum_{q,p} r_qp[a] c_qp[b], r = 4 e_s0 + e_s1 + e_s2,
// c = e_s0 - e_s3 (s_m = kT.v[q][p][m]).  Built at compile time.
struct FormTable {
  int m[6][6];
};
constexpr FormTable make_form_table() {
  FormTable f{};
  for (int q = 0; q < 6; ++q)
    for (int p = 0; p < 6; ++p) {
      const int s0 = kT.v[q][p][0], s1 = kT.v[q][p][1], s2 = kT.v[q][p][2],
                s3 = kT.v[q][p][3];
      const int r[3] = {s0, s1, s2}, rw[3] = {4, 1, 1};
      for (int k = 0; k < 3; ++k) {
        f.m[r[k]][s0] += rw[k];
        f.m[r[k]][s3] -= rw[k];
      }
    }
  return f;
}
constexpr FormTable kM = make_form_table();
template <int A, int B>
struct MM {
  static constexpr int value = kM.m[A][B];
};
// y[B] = sum_A M[A][B] u[A] (zero coefficients fold away)
template <int B, int A = 0>
__device__ __forceinline__ double form_col(const double (&u)[6]) {
  if constexpr (A == 6) {
    return 0.0;
  } else {
    constexpr int c = MM<A, B>::value;
    if constexpr (c == 0) return form_col<B, A + 1>(u);
    else return (double)c * u[A] + form_col<B, A + 1>(u);
  }
}
template <int B = 0>
__device__ __forceinline__ void form_apply(const double (&u)[6], const double (&vd)[6], double &g4,
                                           double &g5) {
  if constexpr (B < 6) {
    const double y = form_col<B>(u);
    g4 += y * u[B];
    g5 += y * vd[B];
    form_apply<B + 1>(u, vd, g4, g5);
  }
}

// a >= b >= c from the flat index n of the set in the order
// (a, then b <= a, then c <= b): n = a(a+1)(a+2)/6 + b(b+1)/2 + c
__device__ __forceinline__ void decode_set(int n, int &a, int &b, int &c) {
  int x = (int)cbrtf(6.0f * (float)n);
  while ((long long)x * (x + 1) * (x + 2) / 6 > n) --x;
  while ((long long)(x + 1) * (x + 2) * (x + 3) / 6 <= n) ++x;
  a = x;
  int r = n - (int)((long long)x * (x + 1) * (x + 2) / 6);
  int y = (int)((sqrtf(8.0f * (float)r + 1.0f) - 1.0f) * 0.5f);
  while (y * (y + 1) / 2 > r) --y;
  while ((y + 1) * (y + 2) / 2 <= r) ++y;
  b = y;
  c = r - y * (y + 1) / 2;
}

// One batch entry's contribution to E[4]T and E[5]ST, every set {a >= b >= c}
// of virtuals evaluated once with all six of its orderings, the distinct
// orderings q of repeated virtuals counted once (a = b keeps q = 0, 1, 4;
// b = c keeps q = 0, 2, 3; a = b = c keeps q = 0).  The loads are staged
// through shared memory.  Block
// (blockIdx.x, blockIdx.y = e) takes one tile triple A >= B >= C of 8-wide
// virtual tiles (decoded like a set) of triplet e and loads, with sector-
// complete row reads, the six permuted 8x8x8 cubes of W (tiles (A,B,C),
// (A,C,B), ..., one per ordering), the 8x8 tiles of the <jk|..>, <ik|..>,
// <ij|..> slabs for every ordered pair of the three tiles, and the t1 rows and
// orbital energies of the three tiles.  Each of its 128 threads then
// evaluates four sets {a >= b >= c} of the cube from shared memory: sets of
// three distinct virtuals through the constant bilinear form, sets with a
// repeated virtual through the general per-ordering sum.
constexpr int kTile = 8;
// kOrd[s][r] in device code: the first position is s / 2, the other two
// follow in increasing order for even s and swapped for odd s
__host__ __device__ __forceinline__ constexpr int ordpos(int s, int r) {
  const int f = s >> 1, lo = f == 0 ? 1 : 0, hi = f == 2 ? 1 : 2;
  return r == 0 ? f : (r == 1 ? ((s & 1) ? hi : lo) : ((s & 1) ? lo : hi));
}
static_assert(ordpos(0, 2) == kOrd[0][2] && ordpos(3, 1) == kOrd[3][1] &&
                  ordpos(4, 2) == kOrd[4][2] && ordpos(5, 0) == kOrd[5][0] &&
                  ordpos(1, 1) == kOrd[1][1] && ordpos(2, 1) == kOrd[2][1],
              "ordpos restates kOrd");
template <typename TW>
__global__ void __launch_bounds__(128)
    k_triples_energy_tiled(const TW *__restrict__ Wbase, long long wstride,
                           const int *__restrict__ trip3, const double *__restrict__ t1,
                           const double *__restrict__ Ioovv, const double *__restrict__ eo,
                           const double *__restrict__ ev, int o, int v,
                           double *__restrict__ part) {
  __shared__ TW cube[6][kTile][kTile + 1][kTile + 1];
  __shared__ double It[3][6][kTile][kTile + 1];
  __shared__ double ts[3][3][kTile];   // [t_i, t_j, t_k][tile position][local]
  __shared__ double es[3][kTile];      // ev of the three tiles
  __shared__ double sh[2][4];
  const int e = blockIdx.y;
  const int i = trip3[3 * e], j = trip3[3 * e + 1], k = trip3[3 * e + 2];
  const TW *__restrict__ W = Wbase + (long long)e * wstride;
  const int mult = (i == j && j == k) ? 6 : ((i == j || j == k) ? 2 : 1);
  const double scale = 1.0 / (3.0 * mult);
  const long long v2 = (long long)v * v;
  int T[3];
  decode_set((int)blockIdx.x, T[0], T[1], T[2]);
  const int b0[3] = {T[0] * kTile, T[1] * kTile, T[2] * kTile};
  const int tid = threadIdx.x;
  // six cubes: cube s spans tiles (T[kOrd[s][0]], T[kOrd[s][1]], T[kOrd[s][2]])
#pragma unroll
  for (int s = 0; s < 6; ++s) {
    const int c0 = b0[ordpos(s, 0)], c1 = b0[ordpos(s, 1)], c2 = b0[ordpos(s, 2)];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = tid + 128 * q;
      const int x = idx >> 6, y = (idx >> 3) & 7, z = idx & 7;
      const int gx = c0 + x, gy = c1 + y, gz = c2 + z;
      cube[s][x][y][z] = (gx < v && gy < v && gz < v) ? W[gx * v2 + (long long)gy * v + gz]
                                                      : (TW)0;
    }
  }
  // integral tiles: slab 0 = <jk|..>, 1 = <ik|..>, 2 = <ij|..>; ordered pair
  // (x, y) of tile positions -> index x * 2 + (y > x ? y - 1 : y)
  const double *slab[3] = {Ioovv + ((long long)j * o + k) * v2, Ioovv + ((long long)i * o + k) * v2,
                           Ioovv + ((long long)i * o + j) * v2};
  for (int idx = tid; idx < 3 * 6 * 64; idx += 128) {
    const int sl = idx / 384, pr = (idx / 64) % 6, r = (idx >> 3) & 7, c = idx & 7;
    const int x = pr >> 1, yy = pr & 1, y = yy < x ? yy : yy + 1;
    const int gr = b0[x] + r, gc = b0[y] + c;
    It[sl][pr][r][c] = (gr < v && gc < v) ? slab[sl][(long long)gr * v + gc] : 0.0;
  }
  if (tid < 72) {
    const int w = tid / 24, pos = (tid / 8) % 3, l = tid & 7;
    const int occ = w == 0 ? i : (w == 1 ? j : k), g = b0[pos] + l;
    ts[w][pos][l] = g < v ? t1[(long long)occ * v + g] : 0.0;
  } else if (tid < 96) {
    const int pos = (tid - 72) / 8, l = tid & 7, g = b0[pos] + l;
    es[pos][l] = g < v ? ev[g] : 0.0;
  }
  __syncthreads();
  const double eijk = eo[i] + eo[j] + eo[k];
  double s4 = 0.0, s5 = 0.0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int n = tid + 128 * q;
    const int l[3] = {n >> 6, (n >> 3) & 7, n & 7};
    const int a = b0[0] + l[0], b = b0[1] + l[1], c = b0[2] + l[2];
    if (a >= v || b >= v || c >= v || a < b || b < c) continue;
    double u[6], vd[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
      const int P0 = ordpos(s, 0), P1 = ordpos(s, 1), P2 = ordpos(s, 2);
      u[s] = (double)cube[s][l[P0]][l[P1]][l[P2]];
      const int p12 = P1 * 2 + (P2 > P1 ? P2 - 1 : P2), p02 = P0 * 2 + (P2 > P0 ? P2 - 1 : P2),
                p01 = P0 * 2 + (P1 > P0 ? P1 - 1 : P1);
      // V - W at (p0,p1,p2): t_i^p0 <jk|p1p2> + t_j^p1 <ik|p0p2> + t_k^p2 <ij|p0p1>
      vd[s] = ts[0][P0][l[P0]] * It[0][p12][l[P1]][l[P2]] +
              ts[1][P1][l[P1]] * It[1][p02][l[P0]][l[P2]] +
              ts[2][P2][l[P2]] * It[2][p01][l[P0]][l[P1]];
    }
    const double D = eijk - es[0][l[0]] - es[1][l[1]] - es[2][l[2]];
    double g4 = 0.0, g5 = 0.0;
    if (a > b && b > c) {
      form_apply(u, vd, g4, g5);
    } else {
      const bool ab = a == b, bc = b == c;
      const bool use[6] = {true, !bc, !ab, !ab, !bc, !(ab || bc)};
      accum_sets<0>(use, u, vd, g4, g5);
    }
    const double inv = 1.0 / D;
    s4 += g4 * inv;
    s5 += g5 * inv;
  }
  for (int off = 16; off; off >>= 1) {
    s4 += __shfl_down_sync(0xffffffffu, s4, off);
    s5 += __shfl_down_sync(0xffffffffu, s5, off);
  }
  const int lane = tid & 31, wid = tid >> 5;
  if (lane == 0) {
    sh[0][wid] = s4;
    sh[1][wid] = s5;
  }
  __syncthreads();
  if (tid == 0) {
    double a4 = 0.0, a5 = 0.0;
    for (int w = 0; w < 4; ++w) {
      a4 += sh[0][w];
      a5 += sh[1][w];
    }
    const long long slot = (long long)e * gridDim.x + blockIdx.x;
    part[2 * slot] = scale * a4;
    part[2 * slot + 1] = scale * a5;
  }
}

// sum of n (E4, E5) partial pairs: 1024 threads stride the list, then a
// fixed-shape tree; the order of additions does not depend on timing
__global__ void __launch_bounds__(1024) k_sum_pairs(double *out, const double *part, long long n) {
  double a = 0.0, b = 0.0;
  for (long long t = threadIdx.x; t < n; t += blockDim.x) {
    a += part[2 * t];
    b += part[2 * t + 1];
  }
  for (int off = 16; off; off >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, off);
    b += __shfl_down_sync(0xffffffffu, b, off);
  }
  __shared__ double sa[32], sb[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { sa[wid] = a; sb[wid] = b; }
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    a = lane < nw ? sa[lane] : 0.0;
    b = lane < nw ? sb[lane] : 0.0;
    for (int off = 16; off; off >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, off);
      b += __shfl_down_sync(0xffffffffu, b, off);
    }
    if (lane == 0) { out[0] = a; out[1] = b; }
  }
}
}  // namespace

// The 12 contractions of a triplet (6 permutations x 2 terms) fall into three
// classes by the position of the virtual that is not a pair index of the
// pair-side operands: class c (W index c on the t2/H side, pairs (a,b)),
// class a (pairs (b,c), index a) and class b (pairs (a,c), index b).  All four
// terms of a class share one output orientation, so each class is ONE
// tensor-core product with four K segments (2 x K = v, 2 x K = o); every
// output view has unit stride along m, the first class stores and the other
// two accumulate with RED.  Per class and segment (P = permutation of (ijk)):
//   class c:  t2[k,i] x Gv[j] (P4)   t2[k,j] x GvT[i] (P5)   -H[j,k] x t2P[i] (P0)   -H[i,k] x t2Q[j] (P2)
//   class a:  Gv[k] x t2[i,j] (P0)   GvT[j] x t2[i,k] (P1)   t2P[j] x -H[k,i] (P3)   t2Q[k] x -H[j,i] (P5)
//   class b:  Gv[k] x t2[j,i] (P2)   GvT[i] x t2[j,k] (P3)   t2P[i] x -H[k,j] (P1)   t2Q[k] x -H[i,j] (P4)
// with Gv[z][(b,c),d] = (bd|cz), GvT[z][(c,b),d] = Gv[z][(b,c),d],
// t2P[x][(a,b),l] = t2[x,l,a,b], t2Q[x][(b,a),l] = t2[x,l,a,b] and
// H[y,z][c,l] = (cz|yl).
//
// Split precision: the triplets run in batches.  Every operand of a class is a
// row window of one of six pre-split parent arrays, so a batch's class is ONE
// persistent tcgen05 launch over the tiles of all its triplets (the triplets'
// windows in a device table, W in FP32 -- below the BF16x3 products' own
// rounding), and one energy launch covers the batch.  The tile order (small
// side, then triplet, then large side) makes the concurrently running CTAs
// share the large operand's rows: a window used by several triplets of the
// batch (Gv[j] for every k of a pair (i,j), Gv[k] across pairs) is read from
// DRAM about once per launch instead of once per triplet.  Four launches per
// batch replace four per triplet.  The FP64 path keeps one triplet at a time.
int CCEngine::triples(double *e4, double *e5, double *seconds, int rank, int nranks) {
  const long long O = o, V = v;
  const long long V2 = V * V, V3 = V * V * V;
  cudaEvent_t t0 = nullptr, t1e = nullptr;
  DBuf Gv, GvT, t2P, t2Q, Hn, Wb, part, outp, dtrip, dent;
  SplitOperand sT2, sGv, sGvT, sHn, sT2P, sT2Q;
  // every exit, the error returns included, gives back the scratch and events
  struct Release {
    std::function<void()> f;
    ~Release() { f(); }
  } release_scratch{[&] {
    for (DBuf *b : {&Gv, &GvT, &t2P, &t2Q, &Hn, &Wb, &part, &outp, &dtrip, &dent}) {
      if (b->p) dev_free(b->p);
      b->p = nullptr;
    }
    for (SplitOperand *sp : {&sT2, &sGv, &sGvT, &sHn, &sT2P, &sT2Q}) {
      if (sp->hi) dev_free(sp->hi);
      sp->hi = sp->lo = nullptr;
    }
    if (t0) cudaEventDestroy(t0);
    if (t1e) cudaEventDestroy(t1e);
  }};
  ACES_CUDA(cudaEventCreate(&t0));
  ACES_CUDA(cudaEventCreate(&t1e));
  ACES_CUDA(cudaEventRecord(t0, st));
  const long long sv[4] = {V * V * V, V * V, V, 1};      // I_ovvv[m,a,e,f]
  const long long s3[4] = {O * O * V, O * V, V, 1};      // I_ooov[m,n,i,e]
  const long long st2[4] = {O * V * V, V * V, V, 1};     // t2[i,j,a,b]
  // Gv[k,b,c,d] = (bd|ck) = <bc|dk> = I_ovvv[k,d,c,b]; GvT[k,c,b,d] = Gv[k,b,c,d]
  ACES_TRY(alloc(Gv, O * V3));
  ACES_TRY(perm(Gv.p, o, v, v, v, 0.0, {PermTerm{I_ovvv.p, 1.0, {sv[0], sv[3], sv[2], sv[1]}}}));
  ACES_TRY(alloc(GvT, O * V3));
  ACES_TRY(perm(GvT.p, o, v, v, v, 0.0, {PermTerm{I_ovvv.p, 1.0, {sv[0], sv[2], sv[3], sv[1]}}}));
  // t2P[i,a,b,l] = t2[i,l,a,b]; t2Q[i,b,a,l] = t2[i,l,a,b]
  ACES_TRY(alloc(t2P, O * O * V2));
  ACES_TRY(perm(t2P.p, o, v, v, o, 0.0, {PermTerm{t2(), 1.0, {st2[0], st2[2], st2[3], st2[1]}}}));
  ACES_TRY(alloc(t2Q, O * O * V2));
  ACES_TRY(perm(t2Q.p, o, v, v, o, 0.0, {PermTerm{t2(), 1.0, {st2[0], st2[3], st2[2], st2[1]}}}));
  // Hn[j,k,c,l] = -(ck|jl) = -I_ooov[l,k,j,c] (the second terms enter with a minus sign)
  ACES_TRY(alloc(Hn, O * O * O * V));
  ACES_TRY(perm(Hn.p, o, o, v, o, 0.0, {PermTerm{I_ooov.p, -1.0, {s3[2], s3[1], s3[3], s3[0]}}}));
  // triplets i >= j >= k of this shard: index t (i, then j <= i, then k <= j)
  // with t % nranks == rank
  std::vector<int> trip;
  long long tix = 0;
  for (int i = 0; i < o; ++i)
    for (int j = 0; j <= i; ++j)
      for (int k = 0; k <= j; ++k, ++tix)
        if (tix % nranks == rank) {
          trip.push_back(i);
          trip.push_back(j);
          trip.push_back(k);
        }
  const int ntrip = (int)trip.size() / 3;
  ACES_TRY(alloc(outp, 2));
  ACES_TRY(alloc(dtrip, (trip.size() + 1) / 2 + 1));
  if (!trip.empty())
    ACES_CUDA(cudaMemcpyAsync(dtrip.p, trip.data(), trip.size() * sizeof(int),
                              cudaMemcpyHostToDevice, st));
  const int *d_trip = reinterpret_cast<const int *>(dtrip.p);
  const bool use_split = prec == ACES_PREC_BF16X3 && v >= 128;
  const CView vc{nullptr, kHugeView, 0, 1, V, V2, V};   // m = c, n = (a,b)
  const CView vcT{nullptr, kHugeView, 0, V, kHugeView, 0, 1};  // m = (a,b), n = c
  const CView va{nullptr, V, V, 1, kHugeView, 0, V2};   // m = (b,c), n = a
  const CView vb{nullptr, V, V2, 1, kHugeView, 0, V};   // m = (a,c), n = b
  long long nparts = 0;

  if (use_split) {
    ACES_TRY(split_pack(sT2, t2(), V, o * o * v, v, st));       // rows (x,y,alpha), K = d
    ACES_TRY(split_pack(sGv, Gv.p, V, o * v * v, v, st));       // rows (z,beta,gamma), K = d
    ACES_TRY(split_pack(sGvT, GvT.p, V, o * v * v, v, st));     // rows (z,gamma,beta), K = d
    ACES_TRY(split_pack(sHn, Hn.p, O, o * o * v, o, st));       // rows (y,z,gamma), K = l
    ACES_TRY(split_pack(sT2P, t2P.p, O, o * v * v, o, st));     // rows (x,alpha,beta), K = l
    ACES_TRY(split_pack(sT2Q, t2Q.p, O, o * v * v, o, st));     // rows (x,beta,alpha), K = l
    // the FP64 copies are not read again
    ACES_CUDA(cudaStreamSynchronize(st));
    for (DBuf *b : {&Gv, &GvT, &t2P, &t2Q}) {
      dev_free(b->p);
      b->p = nullptr;
    }
    // batch size: FP32 W slots within a quarter of the free memory, <= 4 GB
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
      fr = 0;
    }
    const double slot = (double)V3 * sizeof(float);
    const double budget = std::min(0.25 * (double)fr, 4.0e9);
    const int nb = (int)std::max(1.0, std::min((double)std::max(ntrip, 1), budget / slot));
    ACES_TRY(alloc(Wb, (size_t)((V3 * nb + 1) / 2)));  // FP32 slots in a double buffer
    // class c runs transposed on the 128 x 256 tiles (M = (a,b), N = c: the
    // ragged side is the one whose MMA N is cut to the live columns, where on
    // 128-row tiles M = c = v would leave 256 - v rows idle), and stores W
    // rows of v contiguous floats
    const SplitOperand Ac[4] = {sT2, sT2, sHn, sHn}, Bc[4] = {sGv, sGvT, sT2P, sT2Q};
    const bool c_wide = bf16x3_wide_applies(Bc, 4, v);
    // one entry per triplet and class: the windows of the four segments
    auto T2r = [&](int x, int y) { return (x * o + y) * v; };   // rows of sT2 / sHn
    auto Pr = [&](int z) { return z * v * v; };                  // rows of sGv/sGvT/sT2P/sT2Q
    std::vector<BatchEntry> ent((size_t)3 * ntrip);
    for (int t = 0; t < ntrip; ++t) {
      const int i = trip[3 * t], j = trip[3 * t + 1], k = trip[3 * t + 2];
      const long long coff = (long long)(t % nb) * V3;
      BatchEntry &c = ent[(size_t)3 * t], &a = ent[(size_t)3 * t + 1],
                 &b = ent[(size_t)3 * t + 2];
      c = c_wide ? BatchEntry{{Pr(j), Pr(i), Pr(i), Pr(j)},
                              {T2r(k, i), T2r(k, j), T2r(j, k), T2r(i, k)}, coff}
                 : BatchEntry{{T2r(k, i), T2r(k, j), T2r(j, k), T2r(i, k)},
                              {Pr(j), Pr(i), Pr(i), Pr(j)}, coff};
      a = BatchEntry{{Pr(k), Pr(j), Pr(j), Pr(k)},
                     {T2r(i, j), T2r(i, k), T2r(k, i), T2r(j, i)}, coff};
      b = BatchEntry{{Pr(k), Pr(i), Pr(i), Pr(k)},
                     {T2r(j, i), T2r(j, k), T2r(k, j), T2r(i, j)}, coff};
    }
    // entries of class q for triplets [t0, t0 + n) stored contiguously:
    // [class][triplet] on the device
    std::vector<BatchEntry> byclass((size_t)3 * ntrip);
    for (int q = 0; q < 3; ++q)
      for (int t = 0; t < ntrip; ++t) byclass[(size_t)q * ntrip + t] = ent[(size_t)3 * t + q];
    ACES_TRY(alloc(dent, (byclass.size() * sizeof(BatchEntry) + 7) / 8 + 1));
    if (!byclass.empty())
      ACES_CUDA(cudaMemcpyAsync(dent.p, byclass.data(), byclass.size() * sizeof(BatchEntry),
                                cudaMemcpyHostToDevice, st));
    const BatchEntry *d_ent = reinterpret_cast<const BatchEntry *>(dent.p);
    const SplitOperand Aa[4] = {sGv, sGvT, sT2P, sT2Q}, Ba[4] = {sT2, sT2, sHn, sHn};
    const int nt = (v + kTile - 1) / kTile;
    const int nblk = nt * (nt + 1) * (nt + 2) / 6;   // tile triples A >= B >= C
    ACES_TRY(alloc(part, (size_t)std::max(ntrip, 1) * nblk * 2));
    for (int t0b = 0; t0b < ntrip; t0b += nb) {
      const int n = std::min(nb, ntrip - t0b);
      CView cv = c_wide ? vcT : vc;
      cv.p = Wb.p;
      if (c_wide)
        ACES_TRY(gemm_nt_bf16x3_batched(Bc, Ac, 4, v * v, v, &byclass[(size_t)t0b], d_ent + t0b,
                                        n, 1.0, 0.0, cv, true, st));
      else
        ACES_TRY(gemm_nt_bf16x3_batched(Ac, Bc, 4, v, v * v, &byclass[(size_t)t0b],
                                        d_ent + t0b, n, 1.0, 0.0, cv, true, st));
      cv = va;
      cv.p = Wb.p;
      ACES_TRY(gemm_nt_bf16x3_batched(Aa, Ba, 4, v * v, v, &byclass[(size_t)ntrip + t0b],
                                      d_ent + ntrip + t0b, n, 1.0, 1.0, cv, true, st));
      cv = vb;
      cv.p = Wb.p;
      ACES_TRY(gemm_nt_bf16x3_batched(Aa, Ba, 4, v * v, v, &byclass[(size_t)2 * ntrip + t0b],
                                      d_ent + 2 * ntrip + t0b, n, 1.0, 1.0, cv, true, st));
      k_triples_energy_tiled<float><<<dim3(nblk, n), 128, 0, st>>>(
          reinterpret_cast<const float *>(Wb.p), V3, d_trip + 3 * t0b, t1(), I_oovv.p, eo.p,
          ev.p, o, v, part.p + (size_t)t0b * nblk * 2);
      count_launch();
      ACES_CUDA(cudaGetLastError());
    }
    nparts = (long long)ntrip * nblk;
  } else {
    // FP64: one triplet at a time, W in FP64
    ACES_TRY(alloc(Wb, V3));
    const int nt = (v + kTile - 1) / kTile;
    const int nblk = nt * (nt + 1) * (nt + 2) / 6;
    ACES_TRY(alloc(part, (size_t)std::max(ntrip, 1) * nblk * 2));
    auto T2p = [&](int x, int y) { return t2() + ((long long)x * o + y) * V * V; };
    auto Hp = [&](int y, int z) { return Hn.p + ((long long)y * o + z) * V * O; };
    auto Gp = [&](int z) { return Gv.p + (long long)z * V2 * V; };
    auto GTp = [&](int z) { return GvT.p + (long long)z * V2 * V; };
    auto Pp = [&](int x) { return t2P.p + (long long)x * V2 * O; };
    auto Qp = [&](int x) { return t2Q.p + (long long)x * V2 * O; };
    // one class: C(view) = beta C + sum_s A_s B_s^T (K = v for the t2 x (bd|ck)
    // segments, o for the others)
    auto run_class = [&](const double *const (&A)[4], const double *const (&B)[4], int M, int N,
                         const CView &cv, double beta) -> int {
      for (int g = 0; g < 4; ++g) {
        const int K = g < 2 ? v : o;
        ACES_TRY(gemm_nt_f64(M, N, K, 1.0, A[g], K, B[g], K, g == 0 ? beta : 1.0, cv, st));
      }
      return ACES_OK;
    };
    for (int t = 0; t < ntrip; ++t) {
      const int i = trip[3 * t], j = trip[3 * t + 1], k = trip[3 * t + 2];
      CView cv = vc;
      cv.p = Wb.p;
      {
        const double *const A[4] = {T2p(k, i), T2p(k, j), Hp(j, k), Hp(i, k)};
        const double *const B[4] = {Gp(j), GTp(i), Pp(i), Qp(j)};
        ACES_TRY(run_class(A, B, v, v * v, cv, 0.0));
      }
      cv = va;
      cv.p = Wb.p;
      {
        const double *const A[4] = {Gp(k), GTp(j), Pp(j), Qp(k)};
        const double *const B[4] = {T2p(i, j), T2p(i, k), Hp(k, i), Hp(j, i)};
        ACES_TRY(run_class(A, B, v * v, v, cv, 1.0));
      }
      cv = vb;
      cv.p = Wb.p;
      {
        const double *const A[4] = {Gp(k), GTp(i), Pp(i), Qp(k)};
        const double *const B[4] = {T2p(j, i), T2p(j, k), Hp(k, j), Hp(i, j)};
        ACES_TRY(run_class(A, B, v * v, v, cv, 1.0));
      }
      k_triples_energy_tiled<double><<<dim3(nblk, 1), 128, 0, st>>>(
          Wb.p, 0, d_trip + 3 * t, t1(), I_oovv.p, eo.p, ev.p, o, v,
          part.p + (size_t)t * nblk * 2);
      count_launch();
    }
    nparts = (long long)ntrip * nblk;
  }
  k_sum_pairs<<<1, 1024, 0, st>>>(outp.p, part.p, nparts);
  count_launch();
  double h[2];
  ACES_CUDA(cudaMemcpyAsync(h, outp.p, 16, cudaMemcpyDeviceToHost, st));
  ACES_CUDA(cudaEventRecord(t1e, st));
  ACES_CUDA(cudaStreamSynchronize(st));
  if (int tcs = tc_status_and_clear()) {
    set_error("(T): tensor-core contraction gave up waiting (code %d)", tcs);
    return ACES_ERR_TIMEOUT;
  }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, t0, t1e);
  *seconds = ms * 1e-3;
  *e4 = h[0];
  *e5 = h[1];
  if (!std::isfinite(*e4) || !std::isfinite(*e5)) {
    set_error("(T): non-finite energy");
    return ACES_ERR_NAN;
  }
  return ACES_OK;
}

}  // namespace acesb200
