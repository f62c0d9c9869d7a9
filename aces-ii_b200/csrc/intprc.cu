// intprc.cu -- the MO-integral list producer on the device: the six lists the
// closed-shell CC programs read, from density-fitted (or Cholesky) factors of
// the MO two-electron integrals.
//
// The reference's integral chain is vtran (AO -> MO transformation,
// vtran/vtran.F) followed by intprc, which sorts the transformed integrals
// into the irrep-blocked MOINTS lists (intprc/clmoio.F:46-260 creates lists
// 13, 10, 16, 25, 30, 233 with the pair types used here).  This entry point
// takes the MO factors B^L_pq, (pq|rs) = sum_L B^L_pq B^L_rs, and writes each
// list as one FP64 tensor-core product over L:
//
//   list element (row (p,q), column (r,s)) = <pq|rs> = (pr|qs)
//     = sum_L B_RP[r][p][L] B_SQ[s][q][L]
//
// with the K-contiguous factor blocks B_XY[x][y][L] = B^L_{x y} (X, Y the
// occupied or virtual space).  Without symmetry (one irrep) the product is
// written straight into the list's column-major block through a two-level
// output view (m = (r,p) with p fastest has unit stride in the list, so the
// stores coalesce); with irreps it goes to a dense [r][p][s][q] scratch that a
// scatter kernel distributes over the irrep blocks.
#include <vector>

#include "engine.cuh"

using namespace acesb200;

namespace {
struct ListSpec {
  int list, typeL, typeR;
  char P, Q, R, S;
};
// intprc/clmoio.F: list, row pair type, column pair type, index spaces
const ListSpec kLists[6] = {
    {13, 14, 14, 'o', 'o', 'o', 'o'},    // <Ij|Kl>
    {10, 14, 18, 'o', 'o', 'o', 'v'},    // <Ij|Ka>
    {16, 13, 14, 'v', 'v', 'o', 'o'},    // <Ab|Ij>
    {25, 11, 11, 'v', 'o', 'v', 'o'},    // <Ai|Bj>
    {30, 13, 11, 'v', 'v', 'v', 'o'},    // <Ab|Ci>
    {233, 13, 13, 'v', 'v', 'v', 'v'},   // <Ab|Cd>
};
}  // namespace

extern "C" int aces_intprc_df(const double *B, int naux, int on_device) {
  State &stt = state();
  std::lock_guard<std::recursive_mutex> lk(stt.mu);
  const SymInfo &s = stt.sym;
  if (!s.ready) {
    set_error("aces_intprc_df: symmetry not initialised (aces_sym_init)");
    return ACES_ERR_NOSYM;
  }
  if (!B || naux < 1) {
    set_error("aces_intprc_df: null factors or naux %d < 1", naux);
    return ACES_ERR_ARG;
  }
  std::vector<int> irr_o, irr_v;
  for (int h = 0; h < s.nirrep; ++h) {
    for (int k = 0; k < s.pop[h]; ++k) irr_o.push_back(h);
    for (int k = 0; k < s.vrt[h]; ++k) irr_v.push_back(h);
  }
  const long long o = (long long)irr_o.size(), v = (long long)irr_v.size(), n = o + v;
  if (o == 0 || v == 0) {
    set_error("aces_intprc_df: empty occupied or virtual space");
    return ACES_ERR_ARG;
  }
  cudaStream_t st = 0;
  std::vector<void *> owned;
  struct Free {
    std::vector<void *> &p;
    ~Free() {
      cudaStreamSynchronize(0);
      for (void *q : p) dev_free(q);
    }
  } release{owned};
  auto get = [&](double **out, size_t doubles) -> int {
    if (dev_alloc((void **)out, std::max<size_t>(doubles, 1) * 8) != cudaSuccess) {
      cudaGetLastError();
      set_error("aces_intprc_df: device allocation of %zu doubles failed", doubles);
      return ACES_ERR_NOMEM;
    }
    owned.push_back(*out);
    return ACES_OK;
  };
  const double *dB = B;
  if (!on_device) {
    double *t = nullptr;
    ACES_TRY(get(&t, (size_t)naux * n * n));
    ACES_CUDA(cudaMemcpyAsync(t, B, (size_t)naux * n * n * 8, cudaMemcpyHostToDevice, st));
    dB = t;
  }
  // K-contiguous factor blocks XY[x][y][L] = B[L][X0 + x][Y0 + y]
  double *blk[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  const long long dim[2] = {o, v}, off[2] = {0, o};
  for (int X = 0; X < 2; ++X)
    for (int Y = 0; Y < 2; ++Y) {
      ACES_TRY(get(&blk[X][Y], (size_t)(dim[X] * dim[Y] * naux)));
      PermSpec ps;
      ps.n[0] = 1; ps.n[1] = (int)dim[X]; ps.n[2] = (int)dim[Y]; ps.n[3] = naux;
      ps.nterms = 1;
      ps.beta = 0.0;
      ps.t[0].src = dB + off[X] * n + off[Y];
      ps.t[0].alpha = 1.0;
      ps.t[0].s[0] = 0; ps.t[0].s[1] = n; ps.t[0].s[2] = 1; ps.t[0].s[3] = n * n;
      ACES_TRY(permute(blk[X][Y], ps, st));
    }
  auto sp = [](char c) { return c == 'o' ? 0 : 1; };
  double *X = nullptr;
  size_t xcap = 0;
  for (const ListSpec &L : kLists) {
    const long long np = dim[sp(L.P)], nq = dim[sp(L.Q)], nr = dim[sp(L.R)],
                    ns = dim[sp(L.S)];
    const double *A = blk[sp(L.R)][sp(L.P)], *Bm = blk[sp(L.S)][sp(L.Q)];
    const int M = (int)(nr * np), N = (int)(ns * nq);
    DevMap dm;  // touches every irrep of the list (INIPCK), zero-filled
    ACES_TRY(make_map(dm, L.list, L.typeL, L.typeR, irr_o, irr_v, true));
    if (s.nirrep == 1) {
      double *lp = aces_list_devptr(1, L.list);
      const long long nrows = np * nq;
      // m = (r, p), n = (s, q): offset p + q np + (r + s nr) nrows
      const CView C{lp, np, nrows, 1, nq, nr * nrows, np};
      ACES_TRY(gemm_nt_f64(M, N, naux, 1.0, A, naux, Bm, naux, 0.0, C, st));
    } else {
      const size_t need = (size_t)M * N;
      if (need > xcap) {
        ACES_TRY(get(&X, need));
        xcap = need;
      }
      ACES_TRY(gemm_nt_f64(M, N, naux, 1.0, A, naux, Bm, naux, 0.0, cview_rowmajor(X, N), st));
      launch_scatter_rpsq(X, dm.m, st);
      ACES_CUDA(cudaGetLastError());
    }
    ACES_CUDA(cudaStreamSynchronize(st));
  }
  return ACES_OK;
}
