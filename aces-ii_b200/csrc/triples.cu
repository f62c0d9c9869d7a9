// triples.cu -- the (T) correction (trp/trps.F -> trp/trps2.F, trp/d1t2new.F,
// librt3/rmd314.f, trp/e4tijk.F, trp/t1t32n.f) on the device.
//
// For every occupied triplet i >= j >= k the connected triples
//   W_ijk^abc = sum over the 6 simultaneous permutations of (ia)(jb)(kc) of
//     X_ijk^abc = sum_d t(ij,ad) (bd|ck) - sum_l t(il,ab) (ck|jl)
// are built in one v^3 FP64 buffer by 12 contractions whose permuted outputs
// land in place (two-level output views).  The energy kernel then sums, for
// the distinct permutations of (i,j,k) and all orderings of every virtual set
// {a>=b>=c}, the closed-shell expression
//   E[4]T  = 1/3 sum (4W_abc + W_bca + W_cab)(W_abc - W_cba)/D_ijk^abc
//   E[5]ST = 1/3 sum (4W_abc + W_bca + W_cab)(V_abc - V_cba)/D_ijk^abc,
//   V - W = t_i^a (jb|kc) + t_j^b (ia|kc) + t_k^c (ia|jb),
// reading every W element once per triplet.  Partial sums are kept per
// (triplet, block) and reduced in a fixed order: the FP64 energy sum is
// deterministic.
#include <cmath>
#include <vector>

#include "engine.cuh"

namespace acesb200 {

namespace {
// orderings of (a,b,c): 012 021 102 120 201 210
__constant__ int c_T[6][6][4];  // [reorder q][permutation p][abc, bca, cab, cba] -> slot

__global__ void __launch_bounds__(256)
    k_triples_energy(const double *__restrict__ W, const double *__restrict__ t1,
                     const double *__restrict__ Ioovv, const double *__restrict__ eo,
                     const double *__restrict__ ev, int i, int j, int k, int o, int v,
                     double scale, double *__restrict__ part) {
  const long long v2 = (long long)v * v;
  const int ti[3] = {i, j, k};
  double s4 = 0.0, s5 = 0.0;
  const double eijk = eo[i] + eo[j] + eo[k];
  for (int a = blockIdx.x; a < v; a += gridDim.x) {
    const int np = (a + 1) * (a + 1);
    for (int idx = threadIdx.x; idx < np; idx += blockDim.x) {
      const int b = idx / (a + 1), c = idx % (a + 1);
      if (c > b) continue;
      const int x[3] = {a, b, c};
      const int ord[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
      double u[6], vd[6];
#pragma unroll
      for (int s = 0; s < 6; ++s) {
        const int p0 = x[ord[s][0]], p1 = x[ord[s][1]], p2 = x[ord[s][2]];
        u[s] = W[p0 * v2 + (long long)p1 * v + p2];
        // V - W at (p0,p1,p2) for the triplet (i,j,k)
        vd[s] = t1[(long long)ti[0] * v + p0] * Ioovv[(((long long)ti[1] * o + ti[2]) * v + p1) * v + p2] +
                t1[(long long)ti[1] * v + p1] * Ioovv[(((long long)ti[0] * o + ti[2]) * v + p0) * v + p2] +
                t1[(long long)ti[2] * v + p2] * Ioovv[(((long long)ti[0] * o + ti[1]) * v + p0) * v + p1];
      }
      const double D = eijk - ev[a] - ev[b] - ev[c];
      double g4 = 0.0, g5 = 0.0;
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        // skip orderings of (a,b,c) already counted (repeated virtuals)
        bool dup = false;
        for (int q2 = 0; q2 < q; ++q2)
          if (x[ord[q2][0]] == x[ord[q][0]] && x[ord[q2][1]] == x[ord[q][1]] &&
              x[ord[q2][2]] == x[ord[q][2]])
            dup = true;
        if (dup) continue;
#pragma unroll
        for (int pp = 0; pp < 6; ++pp) {
          const int s0 = c_T[q][pp][0], s1 = c_T[q][pp][1], s2 = c_T[q][pp][2],
                    s3 = c_T[q][pp][3];
          const double Z = 4.0 * u[s0] + u[s1] + u[s2];
          g4 += Z * (u[s0] - u[s3]);
          g5 += Z * (vd[s0] - vd[s3]);
        }
      }
      s4 += g4 / D;
      s5 += g5 / D;
    }
  }
  // block reduction (fixed order)
  __shared__ double sh[2][8];
  for (int off = 16; off; off >>= 1) {
    s4 += __shfl_down_sync(0xffffffffu, s4, off);
    s5 += __shfl_down_sync(0xffffffffu, s5, off);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { sh[0][wid] = s4; sh[1][wid] = s5; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a4 = 0.0, a5 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { a4 += sh[0][w]; a5 += sh[1][w]; }
    part[2 * blockIdx.x] = scale * a4;
    part[2 * blockIdx.x + 1] = scale * a5;
  }
}

__global__ void k_sum_pairs(double *out, const double *part, long long n) {
  // one warp, fixed order
  double a = 0.0, b = 0.0;
  for (long long t = threadIdx.x; t < n; t += 32) {
    a += part[2 * t];
    b += part[2 * t + 1];
  }
  for (int off = 16; off; off >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, off);
    b += __shfl_down_sync(0xffffffffu, b, off);
  }
  if (threadIdx.x == 0) { out[0] = a; out[1] = b; }
}

void fill_tables() {
  static bool done = false;
  if (done) return;
  const int O[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  auto index_of = [&](int a, int b, int c) {
    for (int s = 0; s < 6; ++s)
      if (O[s][0] == a && O[s][1] == b && O[s][2] == c) return s;
    return -1;
  };
  const int ARGS[4][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  int S[6][4], COMP[6][6], T[6][6][4];
  for (int p = 0; p < 6; ++p)
    for (int m = 0; m < 4; ++m) {
      int pos[3];
      for (int r = 0; r < 3; ++r) pos[O[p][r]] = ARGS[m][r];
      S[p][m] = index_of(pos[0], pos[1], pos[2]);
    }
  for (int q = 0; q < 6; ++q)
    for (int s = 0; s < 6; ++s) COMP[q][s] = index_of(O[q][O[s][0]], O[q][O[s][1]], O[q][O[s][2]]);
  for (int q = 0; q < 6; ++q)
    for (int p = 0; p < 6; ++p)
      for (int m = 0; m < 4; ++m) T[q][p][m] = COMP[q][S[p][m]];
  cudaMemcpyToSymbol(c_T, T, sizeof(T));
  done = true;
}
}  // namespace

int CCEngine::triples(double *e4, double *e5, double *seconds) {
  const long long O = o, V = v;
  const long long V2 = V * V, V3 = V * V * V;
  fill_tables();
  cudaEvent_t t0, t1e;
  ACES_CUDA(cudaEventCreate(&t0));
  ACES_CUDA(cudaEventCreate(&t1e));
  ACES_CUDA(cudaEventRecord(t0, st));
  const long long sv[4] = {V * V * V, V * V, V, 1};      // I_ovvv[m,a,e,f]
  const long long s3[4] = {O * O * V, O * V, V, 1};      // I_ooov[m,n,i,e]
  const long long st2[4] = {O * V * V, V * V, V, 1};     // t2[i,j,a,b]
  DBuf Gv, t2P, H, Wb, part, outp;
  // Gv[k,b,c,d] = (bd|ck) = <bc|dk> = I_ovvv[k,d,c,b]
  ACES_TRY(alloc(Gv, O * V3));
  ACES_TRY(perm(Gv.p, o, v, v, v, 0.0, {PermTerm{I_ovvv.p, 1.0, {sv[0], sv[3], sv[2], sv[1]}}}));
  // t2P[i,a,b,l] = t2[i,l,a,b]
  ACES_TRY(alloc(t2P, O * O * V2));
  ACES_TRY(perm(t2P.p, o, v, v, o, 0.0, {PermTerm{t2(), 1.0, {st2[0], st2[2], st2[3], st2[1]}}}));
  // H[j,k,c,l] = (ck|jl) = I_ooov[l,k,j,c]
  ACES_TRY(alloc(H, O * O * O * V));
  ACES_TRY(perm(H.p, o, o, v, o, 0.0, {PermTerm{I_ooov.p, 1.0, {s3[2], s3[1], s3[3], s3[0]}}}));
  ACES_TRY(alloc(Wb, V3));
  // triplets i >= j >= k
  std::vector<int> trip;
  for (int i = 0; i < o; ++i)
    for (int j = 0; j <= i; ++j)
      for (int k = 0; k <= j; ++k) { trip.push_back(i); trip.push_back(j); trip.push_back(k); }
  const int ntrip = (int)trip.size() / 3;
  const int nblk = std::min(v, 296);
  ACES_TRY(alloc(part, (size_t)ntrip * nblk * 2));
  ACES_TRY(alloc(outp, 2));
  // split operands of the first-term contractions (constant over triplets)
  const bool use_split = prec == ACES_PREC_BF16X3 && v >= 128;
  SplitOperand sT2, sGv;
  if (use_split) {
    ACES_TRY(split_pack(sT2, t2(), V, o * o * v, v, st));   // rows (x,y,alpha), K = d
    ACES_TRY(split_pack(sGv, Gv.p, V, o * v * v, v, st));   // rows (z,beta,gamma), K = d
  }
  const long long sW[3] = {V2, V, 1};  // W strides of the virtuals paired with i, j, k
  for (int t = 0; t < ntrip; ++t) {
    const int ti[3] = {trip[3 * t], trip[3 * t + 1], trip[3 * t + 2]};
    // the 6 permutations (x,y,z) of positions (0,1,2)
    const int P[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    for (int pp = 0; pp < 6; ++pp) {
      const int px = P[pp][0], py = P[pp][1], pz = P[pp][2];
      const int x = ti[px], y = ti[py], z = ti[pz];
      // first term: C[alpha, (beta,gamma)] = sum_d t2[x,y,alpha,d] Gv[z][(beta,gamma), d]
      CView c1{Wb.p, kHugeView, 0, sW[px], V, sW[py], sW[pz]};
      double beta1 = pp == 0 ? 0.0 : 1.0;
      if (use_split) {
        SplitOperand a = split_view(sT2, (x * o + y) * v, v);
        SplitOperand b = split_view(sGv, z * v * v, v * v);
        ACES_TRY(gemm_nt_bf16x3(a, b, v, v * v, 1.0, beta1, c1, st));
      } else {
        ACES_TRY(gemm_nt_f64(v, v * v, v, 1.0, t2() + ((long long)x * o + y) * V2, V,
                             Gv.p + (long long)z * V3, V, beta1, c1, st));
      }
      // second term: C[(alpha,beta), gamma] -= sum_l t2P[x][(alpha,beta), l] H[y,z][gamma, l]
      CView c2{Wb.p, V, sW[px], sW[py], kHugeView, 0, sW[pz]};
      ACES_TRY(gemm_nt_f64(v * v, v, o, -1.0, t2P.p + (long long)x * V2 * O, O,
                           H.p + ((long long)y * O + z) * V * O, O, 1.0, c2, st));
    }
    int mult = 1;
    if (ti[0] == ti[1] && ti[1] == ti[2]) mult = 6;
    else if (ti[0] == ti[1] || ti[1] == ti[2]) mult = 2;
    k_triples_energy<<<nblk, 256, 0, st>>>(Wb.p, t1(), I_oovv.p, eo.p, ev.p, ti[0], ti[1], ti[2],
                                           o, v, 1.0 / (3.0 * mult),
                                           part.p + (size_t)t * nblk * 2);
    count_launch();
  }
  k_sum_pairs<<<1, 32, 0, st>>>(outp.p, part.p, (long long)ntrip * nblk);
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
  cudaEventDestroy(t0);
  cudaEventDestroy(t1e);
  for (DBuf *b : {&Gv, &t2P, &H, &Wb, &part, &outp}) {
    cudaFree(b->p);
    b->p = nullptr;
  }
  if (sT2.hi) cudaFree(sT2.hi);
  if (sGv.hi) cudaFree(sGv.hi);
  if (!std::isfinite(*e4) || !std::isfinite(*e5)) {
    set_error("(T): non-finite energy");
    return ACES_ERR_NAN;
  }
  return ACES_OK;
}

}  // namespace acesb200
