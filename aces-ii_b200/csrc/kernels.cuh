// kernels.cuh -- launchers of the bandwidth-bound kernels of the CC engine.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace acesb200 {

// ---- resorts ---------------------------------------------------------------
// out[i0,i1,i2,i3] (C order, dims n[0..3]) = beta*out + sum_t alpha[t] *
// in_t[i0*s[t][0] + i1*s[t][1] + i2*s[t][2] + i3*s[t][3]]   (up to 4 terms).
// The index permutations between contractions (libr/sstgen.f, sst02i.f,
// symtr1.F, symrhf.f, spinad1.f, transp.f) are all instances.
struct PermTerm {
  const double *src;
  double alpha;
  long long s[4];
};
struct PermSpec {
  int n[4];
  int nterms;
  PermTerm t[4];
  double beta;
};
int permute(double *out, const PermSpec &spec, cudaStream_t st);
// The same resort (beta = 0, fewer than 2^31 outputs) with the result also
// written as the two BF16 planes (hi, lo; see split_pack) of a contraction
// operand of rows x K, K-contiguous and zero-padded to k_pad: output element
// idx is operand element (idx / K, idx % K).  out may be null (planes only).
int permute_split(double *out, void *hi, void *lo, int K, int k_pad, const PermSpec &spec,
                  cudaStream_t st);

// ---- elementwise -----------------------------------------------------------
// tau = t2 + c * t1[i,a] t1[j,b] over [o,o,v,v] (libr/ftau.f)
void launch_tau(double *tau, const double *t2, const double *t1, double c, int o, int v,
                cudaStream_t st);
// t_new = z / (e_i + e_j - e_a - e_b) (libr2/newt2.F) and t1 = z1/(e_i-e_a) (vcc/e4seng.F);
// z2 is symmetrised in place first (vcc/dodiis0.F SYMETRIZE_T2).
void launch_newt(double *t2n, const double *z2, double *t1n, const double *z1, const double *eo,
                 const double *ev, int o, int v, cudaStream_t st);

// ---- reductions (FP64) --------------------------------------------------------
// partial sums for E_AB = sum tau*V and E_AA' = sum tau*(V - V^T(ab)); out[0..1]
void launch_energy(double *out2, const double *t2, const double *t1, const double *voovv,
                   const double *fov, int o, int v, double *scratch, cudaStream_t st);

// DAMP_CC_RESIDUAL (vcc/damp_cc_residual.F): xn = x + damp (xn - x)
void launch_blend(double *xn, const double *x, double damp, long long n, cudaStream_t st);
// e = xnew - xold (T1 + T2 of a pair-symmetric vector) with, in the same pass,
// absmax_out[0] = its signed absmax over T1, T2(AB) and packed T2(AA) and
// dots_out[k] = <e, hist[k]> over the same three parts (hist[self] is e);
// scratch holds >= 592 * 27 doubles
int launch_diff_stats(double *e, const double *xnew, const double *xold,
                      const double *const *hist, int nh, int self, int o, int v,
                      double *scratch, double *absmax_out, double *dots_out, cudaStream_t st);
// out = sum_k c[k] p[k] over a pair-symmetric [t1 | t2] (c in device memory,
// n <= 25) and absmax_out[0] = its signed absmax over [t1 | t2 | packed AA(t2)]
// (the DIIS residual and its largest element, vcc/dodiis0.F:131-160);
// scratch holds >= 2 * 592 doubles
void launch_lincomb_absmax(double *out, const double *c, const double *const *p, int n, int o,
                           int v, double *scratch, double *absmax_out, cudaStream_t st);
// solve the bordered DIIS system for n <= 25 on the device (libr/dodiis.F);
// B is 25x25 row-major, coef_out[0..n-1]; status_out[0] = 0 ok / 1 singular
void launch_diis_solve(double *coef_out, int *status_out, const double *B, int n, cudaStream_t st);
// out = base + sum_k c[k] * p[k]  (base may be null); with p = stored errors
// this is the DIIS residual, with base = that residual and p = stored iterates
// it is the extrapolated amplitude vector (vcc/dodiis0.F:188-243)
void launch_lincomb(double *out, const double *base, const double *c, const double *const *p,
                    int n, long long len, cudaStream_t st);

// ---- DPD list <-> dense ------------------------------------------------------
// dense[p,q,r,s] for p<np,q<nq,r<nr,s<ns gathered from a list with the given
// row/col pair-index tables (pair index within block, -1 = not stored; sign
// table for antisymmetric packed types), block base pointers and row counts by
// column irrep.
struct DpdMap {
  const int *rowidx;   // [np*nq] pair index of (p,q) or -1
  const int *colidx;   // [nr*ns]
  const signed char *rowsgn;  // [np*nq] +1/-1/0
  const signed char *colsgn;  // [nr*ns]
  const int *irr_p, *irr_q, *irr_r, *irr_s;  // orbital irreps
  double *const *base;  // per column irrep (device array of pointers)
  const int *nrows;     // per column irrep
  int np, nq, nr, ns;
};
void launch_gather(double *dense, const DpdMap &m, cudaStream_t st);
void launch_scatter(const double *dense, const DpdMap &m, cudaStream_t st);
// scatter of X[r][p][s][q] (p, q the row pair, r, s the column pair) into a
// list of FULL pair types
void launch_scatter_rpsq(const double *X, const DpdMap &m, cudaStream_t st);

// packed particle-particle ladder (engine.cu, ladder_packed): pairs[2p], pairs[2p+1]
// = (c, d) of the symmetric pair p (np = v(v+1)/2 of them) followed by the
// antisymmetric pairs (c < d)
void launch_ladder_pack_v(double *Up, double *Um, const double *V, const int *pairs, int v,
                          cudaStream_t st);
// BF16 planes (hi, lo; rows ij k_pad apart) of the packed tau+ / tau- operands
struct LadderPlanes {
  __nv_bfloat16 *hi_p = nullptr, *lo_p = nullptr, *hi_m = nullptr, *lo_m = nullptr;
  int kp_p = 0, kp_m = 0;
};
// tau+ / tau- of the C1 ladder in the packed order p(c,d) = d(d+1)/2 + c,
// m(c,d) = d(d-1)/2 + c (the order of `pairs` in launch_ladder_pack_v); with
// planes: written only as the planes (tp, tm untouched)
void launch_ladder_pack_tau(double *tp, double *tm, const double *tau, int v, int noo,
                            cudaStream_t st, const LadderPlanes *planes = nullptr);
void launch_ladder_unpack(double *Z2, const double *S, const double *A, int v, int noo,
                          cudaStream_t st);

// The same ladder on irrep blocks.  Virtual pairs are ordered by pair irrep g
// (symmetric c <= d and antisymmetric c < d lists, block offsets offP/offM),
// occupied pairs ij by their irrep (list ijs, offsets offIJ, local index ijl);
// U+- are block-diagonal (block g: nP[g]^2 / nM[g]^2 doubles at offUp/offUm)
// and a vector of symmetry hs couples the virtual pairs of irrep g with the
// occupied pairs of irrep g ^ hs (tau blocks nIJ[g ^ hs] x nP[g] at offTp /
// offTm, products S/A with the same sizes, column-major).
struct LadderBlocks {
  int nirrep, hs, o, v;
  int nP[8], nM[8], nIJ[8], offP[9], offM[9], offIJ[9];
  long long offUp[9], offUm[9], offTp[9], offTm[9];
  const int *pp, *mm, *pidx, *midx, *ijs, *ijl, *irr_o, *irr_v;
};
void launch_ladder_pack_v_blk(double *Up, double *Um, const double *V, const LadderBlocks &L,
                              cudaStream_t st);
void launch_ladder_pack_tau_blk(double *tp, double *tm, const double *tau, const LadderBlocks &L,
                                cudaStream_t st);
void launch_ladder_unpack_blk(double *Z2, const double *S, const double *A,
                              const LadderBlocks &L, cudaStream_t st);

}  // namespace acesb200
