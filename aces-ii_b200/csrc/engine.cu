// engine.cu -- closed-shell CCSD on the device: list input, the residual of
// one xvcc iteration (vcc/vcc.F:811-1024) as NT contractions + resorts,
// NEWT2/E4SENG, CMPENG and DIIS (vcc/dodiis0.F) without host round trips
// except the 5 scalars of the convergence test.
//
// Index conventions (C order): t1[i,a]; t2[i,j,a,b] = t_{iJ}^{aB} (the
// reference's list 46, Ab x Ij, in C1); integrals <pq|rs> as I_xxxx[p,q,r,s].
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <utility>

#include "engine.cuh"

namespace acesb200 {

static const long long kHuge = 1LL << 62;

CCEngine::~CCEngine() { release(); }

std::vector<DBuf *> CCEngine::registry() {
  return {&eo, &ev, &foo, &fvv, &fov, &offo, &offv, &fovT, &I_oooo, &I_ooov, &I_oovv,
          &I_ovov, &I_ovvv, &I_vvvv, &L_oovv, &LF, &LovP, &LooP, &LmeP, &I1, &I2, &IvP,
          &IvP2, &IX, &IX2, &WA0, &WB0, &IoP3, &IvT, &IooT, &LT1, &X, &Xn, &Z1,
          &Z2, &tau, &taut, &tautP, &tauT, &U, &Tp, &Tpp, &uT, &wP, &t2P, &Y1, &Y2, &XnP,
          &WA, &WB, &ZT, &XP, &Xmn, &Wmnij, &WmnT, &t1T, &Fae, &Fmi, &Fme, &Fp, &Fpp,
          &FmiT, &FppT, &FmeT, &tmp4, &scratch, &dev_small, &Bmat, &dvec, &L, &Ln, &gE,
          &lrhs, &bwdA, &bwdB, &bwdC, &bwdD, &Up, &Um, &taup, &taum, &Sld, &Ald, &ladpairs, &Ic, &I1n};
}

void CCEngine::release() {
  for (auto &kv : adjoint) if (kv.second.p) dev_free(kv.second.p);
  adjoint.clear();
  for (auto &kv : tcache) if (kv.second.p) dev_free(kv.second.p);
  tcache.clear();
  for (auto &kv : tape_tcache) if (kv.second.p) dev_free(kv.second.p);
  tape_tcache.clear();
  tape.clear();
  active.clear();
  for (DBuf *b : registry()) {
    if (b->p && !b->borrowed) dev_free(b->p);
    b->p = nullptr;
    b->n = 0;
    b->borrowed = false;
  }
  for (auto &b : hx) if (b.p) dev_free(b.p);
  for (auto &b : he) if (b.p) dev_free(b.p);
  hx.clear();
  he.clear();
  for (auto &e : split_cache) {
    if (e.op.hi) dev_free(e.op.hi);
  }
  split_cache.clear();
  if (split_tmpA.hi) dev_free(split_tmpA.hi);
  if (split_tmpB.hi) dev_free(split_tmpB.hi);
  for (auto &t : split_tmpG) {
    if (t.hi) dev_free(t.hi);
    t = SplitOperand();
  }
  split_tmpA = SplitOperand();
  split_tmpB = SplitOperand();
  for (auto &m : memo)
    if (m.op.hi) dev_free(m.op.hi);
  memo.clear();
  memo_on = false;
  if (residual_exec) cudaGraphExecDestroy(residual_exec);
  residual_exec = nullptr;
  if (ev_lad0) cudaEventDestroy(ev_lad0);
  if (ev_lad1) cudaEventDestroy(ev_lad1);
  ev_lad0 = ev_lad1 = nullptr;
  if (st) cudaStreamDestroy(st);
  st = 0;
}

int CCEngine::alloc(DBuf &b, size_t n) {
  if (b.p && b.n >= n) return ACES_OK;
  if (b.borrowed) {
    set_error("engine: a borrowed list buffer cannot be reallocated");
    return ACES_ERR_ARG;
  }
  if (b.p) dev_free(b.p);
  b.p = nullptr;
  b.n = 0;
  size_t bytes = (n ? n : 1) * sizeof(double);
  if (dev_alloc((void **)&b.p, bytes) != cudaSuccess) {
    cudaGetLastError();
    set_error("engine: device allocation of %zu bytes failed", bytes);
    return ACES_ERR_NOMEM;
  }
  b.n = n;
  ACES_CUDA(cudaMemsetAsync(b.p, 0, bytes, st));
  return ACES_OK;
}

int CCEngine::copy(double *dst, const double *src, size_t n) {
  if (recording) {
    TapeOp op;
    op.kind = TapeOp::COPY;
    op.dst = dst;
    op.src = src;
    op.count = n;
    if (is_active(src)) mark_active(dst);
    tape.push_back(op);
  }
  memo_written(dst, (long long)n);
  if (n) ACES_CUDA(cudaMemcpyAsync(dst, src, n * 8, cudaMemcpyDeviceToDevice, st));
  return ACES_OK;
}

CCEngine::MemoEntry &CCEngine::memo_slot(const double *src, long long ld, int rows, int K) {
  for (auto &m : memo)
    if (m.src == src && m.ld == ld && m.rows == rows && m.K == K) return m;
  memo.emplace_back();
  MemoEntry &m = memo.back();
  m.src = src;
  m.ld = ld;
  m.rows = rows;
  m.K = K;
  m.valid = m.fp64 = false;
  return m;
}

// every entry whose FP64 source range overlaps [p, p + n) doubles
void CCEngine::memo_written(const void *p, long long n) {
  if (memo.empty()) return;
  const char *lo = (const char *)p, *hi = lo + n * 8;
  for (auto &m : memo) {
    if (!m.valid) continue;
    const char *a = (const char *)m.src;
    const char *b = a + ((long long)(m.rows - 1) * m.ld + m.K) * 8;
    if (a < hi && lo < b) m.valid = false;
  }
}

// the elements of an M x N view: its extent from the largest offset of each
// dimension ((i / div) * s1 + (i % div) * s0 over i < M or N; strides >= 0)
void CCEngine::memo_written(const CView &C, int M, int N) {
  if (memo.empty() || M <= 0 || N <= 0) return;
  auto span = [](long long div, long long s1, long long s0, int n) {
    if (s1 < 0 || s0 < 0) return -1LL;
    if (div > 0x7fffffff) return (long long)(n - 1) * s0;
    return (long long)((n - 1) / div) * s1 + std::min<long long>(n - 1, div - 1) * s0;
  };
  const long long sm = span(C.mdiv, C.sm1, C.sm0, M), sn = span(C.ndiv, C.sn1, C.sn0, N);
  if (sm < 0 || sn < 0) {
    for (auto &m : memo) m.valid = false;
    return;
  }
  memo_written(C.p, sm + sn + 1);
}

bool CCEngine::fp64_missing(const double *p) const {
  for (const auto &m : memo)
    if (m.valid && !m.fp64 && m.src == p) return true;
  return false;
}

bool CCEngine::splits(int M, int N, long long K) const {
  return prec == ACES_PREC_BF16X3 && M >= 16 && N >= 16 && K >= 128 &&
         (double)M * N * (double)K >= 1.0e8;
}

int CCEngine::perm_split(double *out, int rows, int K, bool consumer_splits, bool keep_fp64,
                         int n0, int n1, int n2, int n3, std::initializer_list<PermTerm> terms) {
  if (!memo_on || recording || !consumer_splits)
    return perm(out, n0, n1, n2, n3, 0.0, terms);
  PermSpec s;
  s.n[0] = n0; s.n[1] = n1; s.n[2] = n2; s.n[3] = n3;
  s.nterms = 0;
  s.beta = 0.0;
  for (const PermTerm &t : terms) s.t[s.nterms++] = t;
  const long long total = (long long)n0 * n1 * n2 * n3;
  if (total != (long long)rows * K) {
    set_error("perm_split: %lld outputs are not %d rows of %d", total, rows, K);
    return ACES_ERR_ARG;
  }
  memo_written(out, total);
  MemoEntry *m = nullptr;
  ACES_TRY(memo_planes(out, rows, K, &m));
  ACES_TRY(permute_split(keep_fp64 ? out : nullptr, m->op.hi, m->op.lo, K, m->op.k_pad, s, st));
  m->valid = true;
  m->fp64 = keep_fp64;
  return ACES_OK;
}

int CCEngine::memo_planes(const double *key, int rows, int K, MemoEntry **out) {
  MemoEntry &m = memo_slot(key, K, rows, K);
  const int kp = (K + kSplitKPad - 1) / kSplitKPad * kSplitKPad;
  const size_t need = (size_t)rows * kp * 2 * 2;
  if (!m.op.hi || m.op.cap < need) {
    if (m.op.hi) dev_free(m.op.hi);
    m.op = SplitOperand();
    ACES_CUDA(dev_alloc(&m.op.hi, need));
    m.op.cap = need;
    ACES_CUDA(cudaMemsetAsync(m.op.hi, 0, need, st));  // the K padding stays zero
  }
  m.op.rows = m.op.rows_pad = rows;
  m.op.k = K;
  m.op.k_pad = kp;
  m.op.lo = (char *)m.op.hi + (size_t)rows * kp * 2;
  *out = &m;
  return ACES_OK;
}

int CCEngine::tau_op(double *out, const double *t2v, const double *t1v, double c) {
  if (recording) {
    TapeOp op;
    op.kind = TapeOp::TAU;
    op.tau = out;
    op.t2 = t2v;
    op.t1 = t1v;
    op.c = c;
    mark_active(out);
    tape.push_back(op);
  }
  memo_written(out, (long long)o * o * v * v);
  launch_tau(out, t2v, t1v, c, o, v, st);
  ACES_CUDA(cudaGetLastError());
  return ACES_OK;
}

int CCEngine::perm(double *out, int n0, int n1, int n2, int n3, double beta,
                   std::initializer_list<PermTerm> terms) {
  PermSpec s;
  s.n[0] = n0; s.n[1] = n1; s.n[2] = n2; s.n[3] = n3;
  s.nterms = 0;
  s.beta = beta;
  for (const PermTerm &t : terms) s.t[s.nterms++] = t;
  if (recording) {
    TapeOp op;
    op.kind = TapeOp::PERM;
    op.out = out;
    op.spec = s;
    bool any = beta != 0.0 && is_active(out);
    for (int t = 0; t < s.nterms; ++t) {
      op.t_act[t] = is_active(s.t[t].src);
      any = any || op.t_act[t];
    }
    if (any) mark_active(out);
    tape.push_back(op);
  }
  memo_written(out, (long long)n0 * n1 * n2 * n3);
  return permute(out, s, st);
}

static PermTerm PT(const double *src, double alpha, long long s0, long long s1, long long s2,
                   long long s3) {
  PermTerm t;
  t.src = src;
  t.alpha = alpha;
  t.s[0] = s0; t.s[1] = s1; t.s[2] = s2; t.s[3] = s3;
  return t;
}

int CCEngine::G(int M, int N, int K, double alpha, const double *A, long long lda, const double *B,
                long long ldb, double beta, const CView &C, bool constA, bool constB) {
  gemm_calls++;
  gemm_flops += 2.0 * M * N * (double)K;
  if (recording) {
    TapeOp op;
    op.kind = TapeOp::GEMM;
    op.M = M; op.N = N; op.K = K;
    op.alpha = alpha; op.beta = beta;
    op.A = A; op.B = B; op.lda = lda; op.ldb = ldb;
    op.C = C;
    op.a_act = is_active(A);
    op.b_act = is_active(B);
    op.c_act = is_active(C.p);
    if (op.a_act || op.b_act) mark_active(C.p);
    tape.push_back(op);
  }
  memo_written(C, M, N);
  // the tensor-core split path: every contraction with K >= 128 and both
  // output dimensions >= 16 (a thin dimension such as nocc is padded to the
  // 128-row tile: the BF16 tensor cores still beat FP64 FMA several-fold);
  // K = nocc products (low-rank updates) stay on the FP64 kernels
  const bool split = splits(M, N, K);
  if (!split && (fp64_missing(A) || fp64_missing(B))) {
    set_error("contraction %d x %d x %d reads an operand held only as split planes", M, N, K);
    return ACES_ERR_ARG;
  }
  // matrix-vector products are bandwidth bound: FP64 GEMV
  if (N == 1) return gemv_f64(M, K, alpha, A, lda, B, beta, C, false, st);
  if (M == 1) return gemv_f64(N, K, alpha, B, ldb, A, beta, C, true, st);
  if (!split) return gemm_nt_f64(M, N, K, alpha, A, lda, B, ldb, beta, C, st);
  // the tensor-core epilogue gives each thread one output row m (consecutive
  // lanes: consecutive m); an output whose unit stride runs along n is
  // computed as C^T = B A^T so that the lanes' stores coalesce
  CView Cv = C;
  if (C.sm0 != 1 && C.sn0 == 1) {
    std::swap(M, N);
    std::swap(A, B);
    std::swap(lda, ldb);
    std::swap(constA, constB);
    Cv = CView{C.p, C.ndiv, C.sn1, C.sn0, C.mdiv, C.sm1, C.sm0};
  }
  const SplitOperand *a = nullptr, *b = nullptr;
  ACES_TRY(split_get(A, lda, M, K, constA, split_tmpA, &a));
  ACES_TRY(split_get(B, ldb, N, K, constB, split_tmpB, &b));
  return gemm_nt_bf16x3(*a, *b, M, N, alpha, beta, Cv, st);
}

int CCEngine::split_get(const double *src, long long ld, int rows, int K, bool cst,
                        SplitOperand &tmp, const SplitOperand **out) {
  if (memo_on && !cst) {
    MemoEntry &m = memo_slot(src, ld, rows, K);
    if (!m.valid) {
      ACES_TRY(split_pack(m.op, src, ld, rows, K, st));
      m.valid = m.fp64 = true;
    }
    *out = &m.op;
    return ACES_OK;
  }
  if (cst) {
    for (auto &e : split_cache)
      if (e.src == src && e.op.rows == rows && e.op.k == K) {
        *out = &e.op;
        return ACES_OK;
      }
    split_cache.emplace_back();
    SplitEntry &e = split_cache.back();
    e.src = src;
    ACES_TRY(split_pack(e.op, src, ld, rows, K, st));
    *out = &e.op;
    return ACES_OK;
  }
  ACES_TRY(split_pack(tmp, src, ld, rows, K, st));
  *out = &tmp;
  return ACES_OK;
}

int CCEngine::Ggroup(const GArgs *g, int n, double beta) {
  bool grouped = prec == ACES_PREC_BF16X3 && !recording && n >= 2 && n <= 3;
  for (int i = 0; i < n && grouped; ++i) grouped = splits(g[i].M, g[i].N, g[i].K);
  if (!grouped) {
    for (int i = 0; i < n; ++i)
      ACES_TRY(G(g[i].M, g[i].N, g[i].K, 1.0, g[i].A, g[i].lda, g[i].B, g[i].ldb, beta, g[i].C,
                 g[i].constA, g[i].constB));
    return ACES_OK;
  }
  const SplitOperand *sa[3], *sb[3];
  GroupedProblem pr[3];
  for (int i = 0; i < n; ++i) memo_written(g[i].C, g[i].M, g[i].N);
  for (int i = 0; i < n; ++i) {
    GArgs q = g[i];
    gemm_calls++;
    gemm_flops += 2.0 * q.M * q.N * (double)q.K;
    if (q.C.sm0 != 1 && q.C.sn0 == 1) {  // coalescing orientation, as in G
      std::swap(q.M, q.N);
      std::swap(q.A, q.B);
      std::swap(q.lda, q.ldb);
      std::swap(q.constA, q.constB);
      q.C = CView{q.C.p, q.C.ndiv, q.C.sn1, q.C.sn0, q.C.mdiv, q.C.sm1, q.C.sm0};
    }
    ACES_TRY(split_get(q.A, q.lda, q.M, q.K, q.constA, split_tmpG[2 * i], &sa[i]));
    ACES_TRY(split_get(q.B, q.ldb, q.N, q.K, q.constB, split_tmpG[2 * i + 1], &sb[i]));
    pr[i].A = sa[i];
    pr[i].B = sb[i];
    pr[i].nseg = 1;
    pr[i].M = q.M;
    pr[i].N = q.N;
    pr[i].C = q.C;
  }
  return gemm_nt_bf16x3_grouped(pr, n, 1.0, beta, st);
}

int CCEngine::Gmulti(int M, int N, const Seg *sg, int nseg, double beta, const CView &C) {
  bool fused = prec == ACES_PREC_BF16X3 && !recording && nseg >= 2 && nseg <= 3;
  for (int i = 0; i < nseg && fused; ++i) fused = splits(M, N, sg[i].K);
  if (!fused) {
    for (int i = 0; i < nseg; ++i)
      ACES_TRY(G(M, N, sg[i].K, 1.0, sg[i].A, sg[i].lda, sg[i].B, sg[i].ldb,
                 i == 0 ? beta : 1.0, C, sg[i].constA, sg[i].constB));
    return ACES_OK;
  }
  memo_written(C, M, N);
  // coalescing orientation as in G: C^T = B A^T when the output's unit stride runs along n
  CView Cv = C;
  const bool swap = C.sm0 != 1 && C.sn0 == 1;
  if (swap) Cv = CView{C.p, C.ndiv, C.sn1, C.sn0, C.mdiv, C.sm1, C.sm0};
  const int Mv = swap ? N : M, Nv = swap ? M : N;
  SplitOperand a[3], b[3];
  for (int i = 0; i < nseg; ++i) {
    gemm_calls++;
    gemm_flops += 2.0 * M * N * (double)sg[i].K;
    const double *pa = swap ? sg[i].B : sg[i].A, *pb = swap ? sg[i].A : sg[i].B;
    const long long la = swap ? sg[i].ldb : sg[i].lda, lb = swap ? sg[i].lda : sg[i].ldb;
    const bool ca = swap ? sg[i].constB : sg[i].constA, cb = swap ? sg[i].constA : sg[i].constB;
    const SplitOperand *sa = nullptr, *sb = nullptr;
    ACES_TRY(split_get(pa, la, Mv, sg[i].K, ca, split_tmpG[2 * i], &sa));
    ACES_TRY(split_get(pb, lb, Nv, sg[i].K, cb, split_tmpG[2 * i + 1], &sb));
    a[i] = *sa;
    b[i] = *sb;
  }
  return gemm_nt_bf16x3_multi(a, b, nseg, Mv, Nv, 1.0, beta, Cv, st);
}

// ---------------------------------------------------------------------------
// list input
// ---------------------------------------------------------------------------
namespace {
struct HostMap {
  std::vector<int> rowidx, colidx;
  std::vector<signed char> rowsgn, colsgn;
};

void pair_table(const SymInfo &s, int type, const std::vector<int> &irr_p,
                const std::vector<int> &loc_p, const std::vector<int> &irr_q,
                const std::vector<int> &loc_q, std::vector<int> &idx,
                std::vector<signed char> &sgn) {
  int np = (int)irr_p.size(), nq = (int)irr_q.size();
  idx.assign((size_t)np * nq, -1);
  sgn.assign((size_t)np * nq, 0);
  PairType t = pair_type(type);
  for (int p = 0; p < np; ++p)
    for (int q = 0; q < nq; ++q) {
      int hp = irr_p[p], hq = irr_q[q], lp = loc_p[p], lq = loc_q[q];
      long long k;
      if (t.packing == 0) {
        idx[(size_t)p * nq + q] = (int)pair_index(s, type, hp, lp, hq, lq);
        sgn[(size_t)p * nq + q] = 1;
      } else if (hp < hq || (hp == hq && lp < lq)) {
        idx[(size_t)p * nq + q] = (int)pair_index(s, type, hp, lp, hq, lq);
        sgn[(size_t)p * nq + q] = 1;
      } else if (hp > hq || (hp == hq && lp > lq)) {
        k = pair_index(s, type, hq, lq, hp, lp);
        idx[(size_t)p * nq + q] = (int)k;
        sgn[(size_t)p * nq + q] = t.packing == 1 ? -1 : 2;  // 2: PCK2 swapped, same value
      }
      // p == q in a PACK type: not stored (zero)
    }
}

template <class T>
int upload(T **d, const std::vector<T> &h) {
  ACES_CUDA(dev_alloc((void **)d, std::max<size_t>(1, h.size()) * sizeof(T)));
  if (!h.empty()) ACES_CUDA(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return ACES_OK;
}

}  // namespace

DevMap::~DevMap() {
  dev_free(d_rowidx); dev_free(d_colidx); dev_free(d_rowsgn); dev_free(d_colsgn);
  for (int k = 0; k < 4; ++k) dev_free(d_irr[k]);
  dev_free(d_base); dev_free(d_nrows);
}

int make_map(DevMap &dm, int list, int typeL, int typeR, const std::vector<int> &irr_o,
             const std::vector<int> &irr_v, bool create) {
  State &stt = state();
  const SymInfo &s = stt.sym;
  auto orbs = [&](char c, std::vector<int> &irr, std::vector<int> &loc) {
    irr = c == 'O' ? irr_o : irr_v;
    loc.resize(irr.size());
    int cnt[8] = {0};
    for (size_t k = 0; k < irr.size(); ++k) loc[k] = cnt[irr[k]]++;
  };
  PairType L = pair_type(typeL), R = pair_type(typeR);
  std::vector<int> ip, lp, iq, lq, ir, lr, is, ls;
  orbs(L.p, ip, lp); orbs(L.q, iq, lq); orbs(R.p, ir, lr); orbs(R.q, is, ls);
  HostMap hm;
  pair_table(s, typeL, ip, lp, iq, lq, hm.rowidx, hm.rowsgn);
  pair_table(s, typeR, ir, lr, is, ls, hm.colidx, hm.colsgn);
  if (create) ACES_TRY(aces_inipck(1, typeL, typeR, list, 1));
  std::vector<double *> base(8, nullptr);
  std::vector<int> nrows(8, 0);
  for (int h = 0; h < s.nirrep; ++h) {
    int nc = 0, nr = 0;
    aces_list_dims(h + 1, list, &nc, &nr);
    if (nc != s.irpdpd[h][typeR - 1] || nr != s.irpdpd[h][typeL - 1]) {
      set_error("list %d irrep %d has %dx%d, expected %dx%d (types %d,%d)", list, h + 1, nr, nc,
                s.irpdpd[h][typeL - 1], s.irpdpd[h][typeR - 1], typeL, typeR);
      return ACES_ERR_NOLIST;
    }
    base[h] = aces_list_devptr(h + 1, list);
    nrows[h] = nr;
  }
  ACES_TRY(upload(&dm.d_rowidx, hm.rowidx));
  ACES_TRY(upload(&dm.d_colidx, hm.colidx));
  ACES_TRY(upload(&dm.d_rowsgn, hm.rowsgn));
  ACES_TRY(upload(&dm.d_colsgn, hm.colsgn));
  ACES_TRY(upload(&dm.d_irr[0], ip));
  ACES_TRY(upload(&dm.d_irr[1], iq));
  ACES_TRY(upload(&dm.d_irr[2], ir));
  ACES_TRY(upload(&dm.d_irr[3], is));
  ACES_TRY(upload(&dm.d_base, base));
  ACES_TRY(upload(&dm.d_nrows, nrows));
  dm.m.rowidx = dm.d_rowidx; dm.m.colidx = dm.d_colidx;
  dm.m.rowsgn = dm.d_rowsgn; dm.m.colsgn = dm.d_colsgn;
  dm.m.irr_p = dm.d_irr[0]; dm.m.irr_q = dm.d_irr[1];
  dm.m.irr_r = dm.d_irr[2]; dm.m.irr_s = dm.d_irr[3];
  dm.m.base = dm.d_base; dm.m.nrows = dm.d_nrows;
  dm.m.np = (int)ip.size(); dm.m.nq = (int)iq.size();
  dm.m.nr = (int)ir.size(); dm.m.ns = (int)is.size();
  return ACES_OK;
}

int CCEngine::load_from_lists() {
  State &stt = state();
  const SymInfo &s = stt.sym;
  if (!s.ready) {
    set_error("xvcc_run: symmetry not initialised (aces_sym_init)");
    return ACES_ERR_NOSYM;
  }
  if (!st) ACES_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  o = v = 0;
  irr_o.clear(); irr_v.clear();
  for (int h = 0; h < s.nirrep; ++h) {
    for (int k = 0; k < s.pop[h]; ++k) irr_o.push_back(h);
    for (int k = 0; k < s.vrt[h]; ++k) irr_v.push_back(h);
    o += s.pop[h];
    v += s.vrt[h];
  }
  nmo = o + v;
  if (o == 0 || v == 0) {
    set_error("xvcc_run: empty occupied or virtual space");
    return ACES_ERR_ARG;
  }
  eps_h.assign(nmo, 0.0);
  ACES_TRY(aces_getrec("SCFEVALA", (long long)nmo * 8, eps_h.data()));
  std::vector<double> F((size_t)nmo * nmo, 0.0);
  nonhf = aces_reclen("FOCKMAT") == (long long)nmo * nmo * 8;
  if (nonhf) {
    ACES_TRY(aces_getrec("FOCKMAT", (long long)nmo * nmo * 8, F.data()));
    for (int p = 0; p < nmo; ++p) eps_h[p] = F[(size_t)p * nmo + p];
  } else {
    for (int p = 0; p < nmo; ++p) F[(size_t)p * nmo + p] = eps_h[p];
  }
  for (double x : eps_h)
    if (!std::isfinite(x)) {
      set_error("xvcc_run: non-finite orbital energy");
      return ACES_ERR_NAN;
    }
  std::vector<double> hoo((size_t)o * o), hvv((size_t)v * v), hov((size_t)o * v),
      hofo((size_t)o * o), hofv((size_t)v * v), hfovT((size_t)v * o);
  for (int i = 0; i < o; ++i)
    for (int j = 0; j < o; ++j) {
      hoo[i * o + j] = F[(size_t)i * nmo + j];
      hofo[i * o + j] = i == j ? 0.0 : F[(size_t)i * nmo + j];
    }
  for (int a = 0; a < v; ++a)
    for (int b = 0; b < v; ++b) {
      hvv[a * v + b] = F[(size_t)(o + a) * nmo + o + b];
      hofv[a * v + b] = a == b ? 0.0 : F[(size_t)(o + a) * nmo + o + b];
    }
  for (int i = 0; i < o; ++i)
    for (int a = 0; a < v; ++a) {
      hov[i * v + a] = F[(size_t)i * nmo + o + a];
      hfovT[a * o + i] = F[(size_t)i * nmo + o + a];
    }
  ACES_TRY(alloc(eo, o)); ACES_TRY(alloc(ev, v));
  ACES_TRY(alloc(foo, (size_t)o * o)); ACES_TRY(alloc(fvv, (size_t)v * v));
  ACES_TRY(alloc(fov, (size_t)o * v)); ACES_TRY(alloc(offo, (size_t)o * o));
  ACES_TRY(alloc(offv, (size_t)v * v)); ACES_TRY(alloc(fovT, (size_t)o * v));
  auto h2d = [&](DBuf &b, const std::vector<double> &h) -> int {
    ACES_CUDA(cudaMemcpyAsync(b.p, h.data(), h.size() * 8, cudaMemcpyHostToDevice, st));
    return ACES_OK;
  };
  std::vector<double> heo(eps_h.begin(), eps_h.begin() + o), hev(eps_h.begin() + o, eps_h.end());
  ACES_TRY(h2d(eo, heo)); ACES_TRY(h2d(ev, hev));
  ACES_TRY(h2d(foo, hoo)); ACES_TRY(h2d(fvv, hvv)); ACES_TRY(h2d(fov, hov));
  ACES_TRY(h2d(offo, hofo)); ACES_TRY(h2d(offv, hofv)); ACES_TRY(h2d(fovT, hfovT));
  ACES_CUDA(cudaStreamSynchronize(st));

  const long long O = o, V = v;
  // list 13 (14,14): <Ij|Kl>  -> I_oooo[i,j,k,l]
  {
    DevMap dm;
    ACES_TRY(make_map(dm, 13, 14, 14, irr_o, irr_v, false));
    ACES_TRY(alloc(I_oooo, O * O * O * O));
    launch_gather(I_oooo.p, dm.m, st);
    ACES_CUDA(cudaStreamSynchronize(st));
  }
  // list 10 (14,18): <Ij|Ka>  -> I_ooov[i,j,k,a]
  {
    DevMap dm;
    ACES_TRY(make_map(dm, 10, 14, 18, irr_o, irr_v, false));
    ACES_TRY(alloc(I_ooov, O * O * O * V));
    launch_gather(I_ooov.p, dm.m, st);
    ACES_CUDA(cudaStreamSynchronize(st));
  }
  // list 16 (13,14): <Ab|Ij> -> dense [a,b,i,j] -> I_oovv[i,j,a,b]
  ACES_TRY(alloc(tmp4, std::max(O * O * V * V, O * V * V * V)));
  {
    DevMap dm;
    ACES_TRY(make_map(dm, 16, 13, 14, irr_o, irr_v, false));
    launch_gather(tmp4.p, dm.m, st);
    ACES_TRY(alloc(I_oovv, O * O * V * V));
    // out (i,j,a,b) <- tmp[a,b,i,j]
    ACES_TRY(perm(I_oovv.p, o, o, v, v, 0.0, {PT(tmp4.p, 1.0, O, 1, V * O * O, O * O)}));
    ACES_CUDA(cudaStreamSynchronize(st));
  }
  // list 25 (11,11): <Ai|Bj> -> dense [a,i,b,j] = <ai|bj>; I_ovov[m,b,j,e] = <mb|je> = <bm|ej> = d[b,m,e,j]
  {
    DevMap dm;
    ACES_TRY(make_map(dm, 25, 11, 11, irr_o, irr_v, false));
    launch_gather(tmp4.p, dm.m, st);
    ACES_TRY(alloc(I_ovov, O * O * V * V));
    // d strides: [a,i,b,j] -> a: O*V*O, i: V*O, b: O, j: 1 ; out (m,b,j,e) = d[b,m,e,j]
    ACES_TRY(perm(I_ovov.p, o, v, o, v, 0.0,
                  {PT(tmp4.p, 1.0, V * O, O * V * O, 1, O)}));
    ACES_CUDA(cudaStreamSynchronize(st));
  }
  // list 30 (13,11): <Ab|Ci> -> dense [a,b,c,i]; I_ovvv[m,a,e,f] = <ma|ef> = <fe|am> = d[f,e,a,m]
  {
    DevMap dm;
    ACES_TRY(make_map(dm, 30, 13, 11, irr_o, irr_v, false));
    launch_gather(tmp4.p, dm.m, st);
    ACES_TRY(alloc(I_ovvv, O * V * V * V));
    // d strides [a,b,c,i]: a: V*V*O, b: V*O, c: O, i: 1; out (m,a,e,f) = d[f,e,a,m]
    ACES_TRY(perm(I_ovvv.p, o, v, v, v, 0.0, {PT(tmp4.p, 1.0, 1, O, V * O, V * V * O)}));
    ACES_CUDA(cudaStreamSynchronize(st));
  }
  // list 233 (13,13): <Ab|Cd> -> I_vvvv[a,b,c,d].  Without symmetry the list
  // block is the full v^2 x v^2 matrix with pair index a + b*v; read as a C
  // array it is L[d][c][b][a] = <ab|cd> = <dc|ba> (real orbitals: bra-ket and
  // electron-label symmetry), i.e. exactly I_vvvv: the engine borrows the
  // list's device memory instead of gathering a second copy (42.5 GB at
  // o = 30, v = 270).
  if (s.nirrep == 1 && aces_isytyp(1, 233) == 13 && aces_isytyp(2, 233) == 13) {
    double *lp = aces_list_devptr(1, 233);
    int nc = 0, nr = 0;
    if (lp && aces_list_dims(1, 233, &nc, &nr) == ACES_OK && (long long)nr == V * V &&
        (long long)nc == V * V) {
      I_vvvv.p = lp;
      I_vvvv.n = (size_t)(V * V) * (V * V);
      I_vvvv.borrowed = true;
      return ACES_OK;
    }
  }
  {
    DevMap dm;
    ACES_TRY(make_map(dm, 233, 13, 13, irr_o, irr_v, false));
    ACES_TRY(alloc(I_vvvv, V * V * V * V));
    launch_gather(I_vvvv.p, dm.m, st);
    ACES_CUDA(cudaStreamSynchronize(st));
  }
  return ACES_OK;
}

// ---------------------------------------------------------------------------
// iteration-independent resorted integrals
// ---------------------------------------------------------------------------
int CCEngine::setup_intermediates() {
  const long long O = o, V = v;
  const long long OV = O * V, OOVV = O * O * V * V, OVVV = O * V * V * V, OOOV = O * O * O * V;
  // strides of the base arrays
  // I_oovv[m,n,e,f]: (O*V*V, V*V, V, 1); I_ovvv[m,a,e,f]: (V*V*V, V*V, V, 1)
  // I_ooov[m,n,i,e]: (O*O*V, O*V, V, 1); I_ovov[m,b,j,e]: (V*O*V, O*V, V, 1)
  const long long so[4] = {O * V * V, V * V, V, 1};
  const long long sv[4] = {V * V * V, V * V, V, 1};
  const long long s3[4] = {O * O * V, O * V, V, 1};
  const long long sj[4] = {V * O * V, O * V, V, 1};
  ACES_TRY(alloc(L_oovv, OOVV));
  ACES_TRY(perm(L_oovv.p, o, o, v, v, 0.0,
                {PT(I_oovv.p, 2.0, so[0], so[1], so[2], so[3]),
                 PT(I_oovv.p, -1.0, so[0], so[1], so[3], so[2])}));
  // LF[a,e,m,f] = 2 I_ovvv[m,a,f,e] - I_ovvv[m,a,e,f]
  ACES_TRY(alloc(LF, OVVV));
  ACES_TRY(perm(LF.p, v, v, o, v, 0.0,
                {PT(I_ovvv.p, 2.0, sv[1], sv[3], sv[0], sv[2]),
                 PT(I_ovvv.p, -1.0, sv[1], sv[2], sv[0], sv[3])}));
  // LovP[e,m,n,f] = L_oovv[m,n,e,f]
  ACES_TRY(alloc(LovP, OOVV));
  ACES_TRY(perm(LovP.p, v, o, o, v, 0.0, {PT(L_oovv.p, 1.0, so[2], so[0], so[1], so[3])}));
  // LooP[m,i,n,e] = 2 I_ooov[m,n,i,e] - I_ooov[n,m,i,e]
  ACES_TRY(alloc(LooP, OOOV));
  ACES_TRY(perm(LooP.p, o, o, o, v, 0.0,
                {PT(I_ooov.p, 2.0, s3[0], s3[2], s3[1], s3[3]),
                 PT(I_ooov.p, -1.0, s3[1], s3[2], s3[0], s3[3])}));
  // LmeP[m,e,n,f] = L_oovv[m,n,e,f]
  ACES_TRY(alloc(LmeP, OOVV));
  ACES_TRY(perm(LmeP.p, o, v, o, v, 0.0, {PT(L_oovv.p, 1.0, so[0], so[2], so[1], so[3])}));
  // I1[m,e,n,f] = I_oovv[m,n,e,f];  I2[m,e,n,f] = I_oovv[m,n,f,e]
  ACES_TRY(alloc(I1, OOVV));
  ACES_TRY(perm(I1.p, o, v, o, v, 0.0, {PT(I_oovv.p, 1.0, so[0], so[2], so[1], so[3])}));
  ACES_TRY(alloc(I2, OOVV));
  ACES_TRY(perm(I2.p, o, v, o, v, 0.0, {PT(I_oovv.p, 1.0, so[0], so[3], so[1], so[2])}));
  // Ic = I1 - I2 / 2, I1n = -I1: W(mbej) += Y2 Ic^T + XnP I1n^T (one launch)
  ACES_TRY(alloc(Ic, OOVV));
  ACES_TRY(perm(Ic.p, o, v, o, v, 0.0,
                {PT(I_oovv.p, 1.0, so[0], so[2], so[1], so[3]),
                 PT(I_oovv.p, -0.5, so[0], so[3], so[1], so[2])}));
  ACES_TRY(alloc(I1n, OOVV));
  ACES_TRY(perm(I1n.p, o, v, o, v, 0.0, {PT(I_oovv.p, -1.0, so[0], so[2], so[1], so[3])}));
  // IvP[b,m,e,f] = I_ovvv[m,b,e,f]; IvP2[b,m,e,f] = I_ovvv[m,b,f,e]
  ACES_TRY(alloc(IvP, OVVV));
  ACES_TRY(perm(IvP.p, v, o, v, v, 0.0, {PT(I_ovvv.p, 1.0, sv[1], sv[0], sv[2], sv[3])}));
  ACES_TRY(alloc(IvP2, OVVV));
  ACES_TRY(perm(IvP2.p, v, o, v, v, 0.0, {PT(I_ovvv.p, 1.0, sv[1], sv[0], sv[3], sv[2])}));
  // IX[j,m,e,n] = I_ooov[n,m,j,e]; IX2[j,m,e,n] = I_ooov[m,n,j,e]
  ACES_TRY(alloc(IX, OOOV));
  ACES_TRY(perm(IX.p, o, o, v, o, 0.0, {PT(I_ooov.p, 1.0, s3[2], s3[1], s3[3], s3[0])}));
  ACES_TRY(alloc(IX2, OOOV));
  ACES_TRY(perm(IX2.p, o, o, v, o, 0.0, {PT(I_ooov.p, 1.0, s3[2], s3[0], s3[3], s3[1])}));
  // WA0[j,b,m,e] = <mb|ej> = I_oovv[m,j,e,b];  WB0[j,b,m,e] = -<mb|je> = -I_ovov[m,b,j,e]
  ACES_TRY(alloc(WA0, OOVV));
  ACES_TRY(perm(WA0.p, o, v, o, v, 0.0, {PT(I_oovv.p, 1.0, so[1], so[3], so[0], so[2])}));
  ACES_TRY(alloc(WB0, OOVV));
  ACES_TRY(perm(WB0.p, o, v, o, v, 0.0, {PT(I_ovov.p, -1.0, sj[2], sj[1], sj[0], sj[3])}));
  // IoP3[i,j,b,m] = I_ooov[i,j,m,b]
  ACES_TRY(alloc(IoP3, OOOV));
  ACES_TRY(perm(IoP3.p, o, o, v, o, 0.0, {PT(I_ooov.p, 1.0, s3[0], s3[1], s3[3], s3[2])}));
  // IvT[j,a,b,e] = I_ovvv[j,e,b,a]
  ACES_TRY(alloc(IvT, OVVV));
  ACES_TRY(perm(IvT.p, o, v, v, v, 0.0, {PT(I_ovvv.p, 1.0, sv[0], sv[3], sv[2], sv[1])}));
  // IooT[i,m,n,e] = I_ooov[m,n,i,e]
  ACES_TRY(alloc(IooT, OOOV));
  ACES_TRY(perm(IooT.p, o, o, o, v, 0.0, {PT(I_ooov.p, 1.0, s3[2], s3[0], s3[1], s3[3])}));
  // LT1[i,a,n,f] = 2<na|fi> - <na|if> = 2 I_oovv[n,i,f,a] - I_ovov[n,a,i,f]
  ACES_TRY(alloc(LT1, OOVV));
  ACES_TRY(perm(LT1.p, o, v, o, v, 0.0,
                {PT(I_oovv.p, 2.0, so[1], so[3], so[0], so[2]),
                 PT(I_ovov.p, -1.0, sj[2], sj[1], sj[0], sj[3])}));
  // working storage
  ACES_TRY(alloc(X, OV + OOVV));
  ACES_TRY(alloc(Xn, OV + OOVV));
  ACES_TRY(alloc(Z1, OV));
  ACES_TRY(alloc(Z2, OOVV));
  DBuf *big[] = {&tau, &taut, &tautP, &tauT, &U, &Tp, &Tpp, &uT, &wP, &t2P,
                 &Y1, &Y2, &XnP, &WA, &WB, &XP};
  for (DBuf *b : big) ACES_TRY(alloc(*b, OOVV));
  ACES_TRY(alloc(ZT, OOOV));
  ACES_TRY(alloc(Xmn, O * O * O * O));
  ACES_TRY(alloc(Wmnij, O * O * O * O));
  ACES_TRY(alloc(WmnT, O * O * O * O));
  ACES_TRY(alloc(t1T, OV));
  ACES_TRY(alloc(Fae, V * V)); ACES_TRY(alloc(Fp, V * V));
  ACES_TRY(alloc(Fmi, O * O)); ACES_TRY(alloc(Fpp, O * O));
  ACES_TRY(alloc(FmiT, O * O)); ACES_TRY(alloc(FppT, O * O));
  ACES_TRY(alloc(Fme, OV)); ACES_TRY(alloc(FmeT, OV));
  ACES_TRY(alloc(scratch, 592 * 32));
  ACES_TRY(alloc(dev_small, 64 + 25 * 25 + 32));
  ACES_TRY(alloc(Bmat, 25 * 25));
  ACES_CUDA(cudaStreamSynchronize(st));
  // tmp4 is no longer needed
  if (tmp4.p) { dev_free(tmp4.p); tmp4.p = nullptr; tmp4.n = 0; }
  return ACES_OK;
}

int CCEngine::read_guess(bool *read) {
  *read = false;
  const SymInfo &s = state().sym;
  // both lists present with this system's pair types, irrep by irrep
  for (int h = 0; h < s.nirrep; ++h) {
    int nc = 0, nr = 0;
    if (aces_list_dims(h + 1, 46, &nc, &nr) != ACES_OK || nc != s.irpdpd[h][13] ||
        nr != s.irpdpd[h][12]) {
      cudaGetLastError();
      return ACES_OK;
    }
  }
  int nc9 = 0, nr9 = 0;
  if (aces_list_dims(1, 90, &nc9, &nr9) != ACES_OK || nc9 < 1 || nr9 != s.irpdpd[0][8])
    return ACES_OK;
  const long long O = o, V = v;
  // list 46 (13,14) -> dense [a,b,i,j] -> t2[i,j,a,b]
  DBuf tmpb;
  ACES_TRY(alloc(tmpb, O * O * V * V));
  {
    DevMap dm;
    ACES_TRY(make_map(dm, 46, 13, 14, irr_o, irr_v, false));
    launch_gather(tmpb.p, dm.m, st);
    ACES_CUDA(cudaStreamSynchronize(st));
  }
  ACES_TRY(perm(t2(), o, o, v, v, 0.0, {PT(tmpb.p, 1.0, O, 1, V * O * O, O * O)}));
  // list 90 irrep 1: one column over the (a,i) pairs of type 9
  std::vector<double> col((size_t)nr9), h1((size_t)o * v, 0.0);
  ACES_TRY(aces_getlst(col.data(), 1, 1, 1, 90));
  std::vector<int> lo(o), lv(v);
  int cnt[8] = {0};
  for (int i = 0; i < o; ++i) lo[i] = cnt[irr_o[i]]++;
  for (int k = 0; k < 8; ++k) cnt[k] = 0;
  for (int a = 0; a < v; ++a) lv[a] = cnt[irr_v[a]]++;
  for (int i = 0; i < o; ++i)
    for (int a = 0; a < v; ++a)
      if (irr_o[i] == irr_v[a])
        h1[(size_t)i * v + a] = col[pair_index(s, 9, irr_v[a], lv[a], irr_o[i], lo[i])];
  ACES_CUDA(cudaMemcpyAsync(t1(), h1.data(), h1.size() * 8, cudaMemcpyHostToDevice, st));
  ACES_CUDA(cudaStreamSynchronize(st));
  dev_free(tmpb.p);
  *read = true;
  return ACES_OK;
}

int CCEngine::mp2_guess() {
  // T2 = <ij|ab>/D, T1 = 0 (intprc FORMT2)
  ACES_CUDA(cudaMemsetAsync(Z1.p, 0, (size_t)o * v * 8, st));
  launch_newt(t2(), I_oovv.p, t1(), Z1.p, eo.p, ev.p, o, v, st);
  ACES_CUDA(cudaGetLastError());
  return ACES_OK;
}

// ---------------------------------------------------------------------------
// the residual of one CCSD iteration: Z1, Z2 from X = [t1 | t2]
// ---------------------------------------------------------------------------
int CCEngine::residual() {
  // split planes of the pass's non-constant operands are shared between its
  // contractions (and written by the resorts that produce them) only inside
  // this pass; every entry starts invalid
  for (auto &m : memo) m.valid = false;
  struct MemoScope {
    CCEngine &E;
    explicit MemoScope(CCEngine &e) : E(e) {
      E.memo_on = !E.recording && E.prec == ACES_PREC_BF16X3;
    }
    ~MemoScope() {
      E.memo_on = false;
      for (auto &m : E.memo) m.valid = false;
    }
  } memo_scope(*this);
  const long long O = o, V = v;
  const long long OV = O * V, VV = V * V, OO = O * O, OVV = O * V * V, OOV = O * O * V;
  double *T1 = t1(), *T2 = t2();
  const long long st2[4] = {O * V * V, V * V, V, 1};  // t2[i,j,a,b]
  // t1T[a,m]
  ACES_TRY(perm(t1T.p, 1, 1, v, o, 0.0, {PT(T1, 1.0, 0, 0, 1, V)}));
  // FTAU (libr/ftau.f)
  ACES_TRY(tau_op(tau.p, T2, T1, 1.0));
  ACES_TRY(tau_op(taut.p, T2, T1, 0.5));
  // ---- F(ae): QUAD3 + T1RING (vcc/quad3.f, libr/t1ring.F) ----
  ACES_TRY(copy(Fae.p, offv.p, VV));
  ACES_TRY(G(v, v, o, -0.5, t1T.p, O, fovT.p, O, 1.0, cview_rowmajor(Fae.p, V)));
  ACES_TRY(G(v * v, 1, o * v, 1.0, LF.p, OV, T1, OV, 1.0, cview_rowmajor(Fae.p, 1), true));
  // tautP[a,m,n,f] = taut[m,n,a,f]
  ACES_TRY(perm_split(tautP.p, v, o * o * v, splits(v, v, OOV), false, v, o, o, v,
                      {PT(taut.p, 1.0, st2[2], st2[0], st2[1], st2[3])}));
  ACES_TRY(G(v, v, o * o * v, -1.0, tautP.p, OOV, LovP.p, OOV, 1.0, cview_rowmajor(Fae.p, V),
             false, true));
  // ---- F(mi): QUAD2 + T1INW2 (vcc/quad2.f, vcc/t1inw2.f) ----
  ACES_TRY(copy(Fmi.p, offo.p, OO));
  ACES_TRY(G(o, o, v, 0.5, fov.p, V, T1, V, 1.0, cview_rowmajor(Fmi.p, O)));
  ACES_TRY(G(o * o, 1, o * v, 1.0, LooP.p, OV, T1, OV, 1.0, cview_rowmajor(Fmi.p, 1), true));
  ACES_TRY(G(o, o, o * v * v, 1.0, L_oovv.p, OVV, taut.p, OVV, 1.0, cview_rowmajor(Fmi.p, O),
             true));
  // ---- F(me): MAKFME (vcc/makfme.F) ----
  ACES_TRY(copy(Fme.p, fov.p, OV));
  ACES_TRY(G(o * v, 1, o * v, 1.0, LmeP.p, OV, T1, OV, 1.0, cview_rowmajor(Fme.p, 1), true));
  // F'(be) = F(be) - 1/2 t(mb) F(me);  F''(mj) = F(mj) + 1/2 F(me) t(je)
  ACES_TRY(perm(FmeT.p, 1, 1, v, o, 0.0, {PT(Fme.p, 1.0, 0, 0, 1, V)}));
  ACES_TRY(copy(Fp.p, Fae.p, VV));
  ACES_TRY(G(v, v, o, -0.5, t1T.p, O, FmeT.p, O, 1.0, cview_rowmajor(Fp.p, V)));
  ACES_TRY(copy(Fpp.p, Fmi.p, OO));
  ACES_TRY(G(o, o, v, 0.5, Fme.p, V, T1, V, 1.0, cview_rowmajor(Fpp.p, O)));
  ACES_TRY(perm(FppT.p, 1, 1, o, o, 0.0, {PT(Fpp.p, 1.0, 0, 0, 1, O)}));
  ACES_TRY(perm(FmiT.p, 1, 1, o, o, 0.0, {PT(Fmi.p, 1.0, 0, 0, 1, O)}));

  // ---- T1 increments (INITSN, FEACONT, FMICONT, FMECONT, T1INT1, E4S) ----
  ACES_TRY(copy(Z1.p, fov.p, OV));
  ACES_TRY(G(o, v, v, 1.0, T1, V, Fae.p, V, 1.0, cview_rowmajor(Z1.p, V)));
  ACES_TRY(G(o, v, o, -1.0, FmiT.p, O, t1T.p, O, 1.0, cview_rowmajor(Z1.p, V)));
  // U[i,a,m,e] = 2 t2[i,m,a,e] - t2[m,i,a,e]
  ACES_TRY(perm_split(U.p, o * v, o * v, splits(o * v, o * v, OV), true, o, v, o, v,
                      {PT(T2, 2.0, st2[0], st2[2], st2[1], st2[3]),
                       PT(T2, -1.0, st2[1], st2[2], st2[0], st2[3])}));
  ACES_TRY(G(o * v, 1, o * v, 1.0, U.p, OV, Fme.p, OV, 1.0, cview_rowmajor(Z1.p, 1)));
  ACES_TRY(G(o * v, 1, o * v, 1.0, LT1.p, OV, T1, OV, 1.0, cview_rowmajor(Z1.p, 1), true));
  // T2T1AB1: wP[i,m,e,f] = 2 t2[i,m,f,e] - t2[i,m,e,f];  Z1[i,a] += sum IvP[a,(mef)] wP[i,(mef)]
  // (IvP[a,m,e,f] = <ma|ef>)
  ACES_TRY(perm_split(wP.p, o, o * v * v, splits(v, o, OVV), false, o, o, v, v,
                      {PT(T2, 2.0, st2[0], st2[1], st2[3], st2[2]),
                       PT(T2, -1.0, st2[0], st2[1], st2[2], st2[3])}));
  ACES_TRY(G(v, o, o * v * v, 1.0, IvP.p, OVV, wP.p, OVV, 1.0, cview_colmajor(Z1.p, V), true));
  // T2T1AB2: uT[a,m,n,e] = 2 t2[m,n,a,e] - t2[n,m,a,e];  Z1[i,a] -= sum uT[a,(mne)] IooT[i,(mne)]
  ACES_TRY(perm_split(uT.p, v, o * o * v, splits(v, o, OOV), false, v, o, o, v,
                      {PT(T2, 2.0, st2[2], st2[0], st2[1], st2[3]),
                       PT(T2, -1.0, st2[2], st2[1], st2[0], st2[3])}));
  ACES_TRY(G(v, o, o * o * v, -1.0, uT.p, OOV, IooT.p, OOV, 1.0, cview_colmajor(Z1.p, V), false,
             true));

  // ---- W(mnij) (QUAD1, T1INW2) and the hole-hole ladder (DRLAD ITYPE=1) ----
  ACES_TRY(G(o * o * o, o, v, 1.0, I_ooov.p, V, T1, V, 0.0, cview_rowmajor(Xmn.p, O), true));
  const long long s4[4] = {O * O * O, O * O, O, 1};
  ACES_TRY(perm(Wmnij.p, o, o, o, o, 0.0,
                {PT(I_oooo.p, 1.0, s4[0], s4[1], s4[2], s4[3]),
                 PT(Xmn.p, 1.0, s4[0], s4[1], s4[2], s4[3]),
                 PT(Xmn.p, 1.0, s4[1], s4[0], s4[3], s4[2])}));
  ACES_TRY(G(o * o, o * o, v * v, 1.0, I_oovv.p, VV, tau.p, VV, 1.0,
             cview_rowmajor(Wmnij.p, OO), true));
  ACES_TRY(perm(WmnT.p, 1, 1, o * o, o * o, 0.0, {PT(Wmnij.p, 1.0, 0, 0, 1, OO)}));
  // INITIN: Z2 <- <ij|ab>
  ACES_TRY(copy(Z2.p, I_oovv.p, (size_t)OO * VV));
  // tauT[a,b,m,n] = tau[m,n,a,b]
  ACES_TRY(perm_split(tauT.p, v * v, o * o, splits(v * v, o * o, OO), false, v, v, o, o,
                      {PT(tau.p, 1.0, st2[2], st2[3], st2[0], st2[1])}));
  ACES_TRY(G(v * v, o * o, o * o, 1.0, tauT.p, OO, WmnT.p, OO, 1.0, cview_colmajor(Z2.p, VV)));
  // ---- particle-particle ladder (DRLAD ITYPE=6, vcc/ladab1.F:61) ----
  if (!ev_lad0) {
    ACES_CUDA(cudaEventCreate(&ev_lad0));
    ACES_CUDA(cudaEventCreate(&ev_lad1));
  }
  // inside a graph capture the records become external event nodes, which
  // record the events again on every replay (the ladder stays timed)
  const unsigned evflag = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
  ACES_CUDA(cudaEventRecordWithFlags(ev_lad0, st, evflag));
  if (recording) {
    // one tape entry for the whole ladder: its adjoint is the same packed
    // ladder applied to the output's adjoint (<ab|cd> = <cd|ab>)
    TapeOp op;
    op.kind = TapeOp::LADDER;
    op.src = tau.p;
    op.dst = Z2.p;
    if (is_active(tau.p)) mark_active(Z2.p);
    tape.push_back(op);
  }
  {
    const bool rec = recording;
    recording = false;  // the ladder's own products and kernels are not taped
    const int ls = ladder_packed(tau.p, Z2.p);
    recording = rec;
    ACES_TRY(ls);
  }
  ACES_CUDA(cudaEventRecordWithFlags(ev_lad1, st, evflag));

  // ---- W(mbej) ABAB and ABBA (DWMBEJ, T1RING), layout W[j,b,m,e] ----
  ACES_TRY(copy(WA.p, WA0.p, (size_t)OO * VV));
  ACES_TRY(G(o, o * v * v, v, 1.0, T1, V, IvP.p, V, 1.0, cview_rowmajor(WA.p, OVV), false, true));
  CView vWn{WA.p, kHuge, 0, OV, OV, OVV, 1};
  ACES_TRY(G(v, o * o * v, o, -1.0, t1T.p, O, IX.p, O, 1.0, vWn, false, true));
  // Y2[j,b,n,f] = t2[n,j,f,b];  XnP[j,b,n,f] = 1/2 t2[j,n,f,b] + t1[j,f] t1[n,b]; Y1 = Y2 - XnP
  ACES_TRY(perm_split(Y2.p, o * v, o * v, splits(o * v, o * v, OV), false, o, v, o, v,
                      {PT(T2, 1.0, st2[1], st2[3], st2[0], st2[2])}));
  ACES_TRY(perm(XnP.p, o, v, o, v, 0.0, {PT(T2, 0.5, st2[0], st2[3], st2[1], st2[2])}));
  // + t1[j,f] t1[n,b]: rank-1 per (j,b,n,f) -> GEMM over a unit K: A[(j),f]... use outer product
  {
    // XnP[j,b,n,f] += t1[j,f] t1[n,b]: a K = 1 product C[(j,f),(n,b)] written through the view
    CView vx{XnP.p, V, OVV, 1, V, V, OV};
    ACES_TRY(G(o * v, o * v, 1, 1.0, T1, 1, T1, 1, 1.0, vx));
  }
  // WA += (Y2 - XnP) I1^T - 1/2 Y2 I2^T = Y2 Ic^T + XnP I1n^T: one two-segment launch
  {
    const Seg sgw[2] = {{Y2.p, OV, Ic.p, OV, o * v, false, true},
                        {XnP.p, OV, I1n.p, OV, o * v, false, true}};
    ACES_TRY(Gmulti(o * v, o * v, sgw, 2, 1.0, cview_rowmajor(WA.p, OV)));
  }
  ACES_TRY(copy(WB.p, WB0.p, (size_t)OO * VV));
  ACES_TRY(G(o, o * v * v, v, -1.0, T1, V, IvP2.p, V, 1.0, cview_rowmajor(WB.p, OVV), false, true));
  CView vWn2{WB.p, kHuge, 0, OV, OV, OVV, 1};
  ACES_TRY(G(v, o * o * v, o, 1.0, t1T.p, O, IX2.p, O, 1.0, vWn2, false, true));
  ACES_TRY(G(o * v, o * v, o * v, 1.0, XnP.p, OV, I2.p, OV, 1.0, cview_rowmajor(WB.p, OV), false,
             true));

  // ---- terms symmetrised by P(ia,jb), accumulated in XP[i,j,a,b] ----
  // FEACONT (vcc/feacont.f)
  ACES_TRY(G(o * o * v, v, v, 1.0, T2, V, Fp.p, V, 0.0, cview_rowmajor(XP.p, V)));
  // FMICONT (vcc/fmicont.f): t2P[i,a,b,m] = t2[i,m,a,b]
  ACES_TRY(perm(t2P.p, o, v, v, o, 0.0, {PT(T2, 1.0, st2[0], st2[2], st2[3], st2[1])}));
  CView vfm{XP.p, VV, OVV, 1, kHuge, 0, VV};
  ACES_TRY(G(o * v * v, o, o, -1.0, t2P.p, O, FppT.p, O, 1.0, vfm));
  // ZT[i,j,b,m] = <mb|ij> + sum_ef <mb|ef> tau(ij,ef) + sum_e <mb|ej> t(ie) + sum_e <mb|ie> t(je)
  // (T1INT2A, T1INW1, T12INT2), then XP -= sum_m t(ma) ZT[(ijb), m].  The
  // tau product runs over the rows (b, m) of IvP[b,m,e,f] = <mb|ef>, the
  // order of ZT's (b, m): unit stride along the product's rows.
  ACES_TRY(copy(ZT.p, IoP3.p, (size_t)OOV * O));
  ACES_TRY(G(o * v, o * o, v * v, 1.0, IvP.p, VV, tau.p, VV, 1.0, cview_colmajor(ZT.p, OV),
             true));
  ACES_TRY(G(o * v * o, o, v, 1.0, WA0.p, V, T1, V, 1.0, cview_colmajor(ZT.p, OOV), true));
  CView vz3{ZT.p, V * O, OOV, 1, kHuge, 0, V * O};
  ACES_TRY(G(o * v * o, o, v, -1.0, WB0.p, V, T1, V, 1.0, vz3, true));
  CView vxp{XP.p, V, VV, 1, kHuge, 0, V};
  ACES_TRY(G(o * o * v, v, o, -1.0, ZT.p, O, t1T.p, O, 1.0, vxp));
  // T1INT2B (vcc/t1int2b.f)
  ACES_TRY(G(o, o * v * v, v, 1.0, T1, V, IvT.p, V, 1.0, cview_rowmajor(XP.p, OVV), false, true));
  // ring (DRRNG/RNGDRV, vcc/rngdrv.f): Tp[i,a,m,e] = t2[i,m,a,e]; Tpp[j,a,m,e] = t2[j,m,e,a]
  ACES_TRY(perm_split(Tp.p, o * v, o * v, splits(o * v, o * v, OV), false, o, v, o, v,
                      {PT(T2, 1.0, st2[0], st2[2], st2[1], st2[3])}));
  ACES_TRY(perm_split(Tpp.p, o * v, o * v, splits(o * v, o * v, OV), false, o, v, o, v,
                      {PT(T2, 1.0, st2[0], st2[3], st2[1], st2[2])}));
  CView vr1{XP.p, V, OVV, V, V, VV, 1};
  {
    const Seg sgr[2] = {{U.p, OV, WA.p, OV, o * v, false, false},
                        {Tp.p, OV, WB.p, OV, o * v, false, false}};
    ACES_TRY(Gmulti(o * v, o * v, sgr, 2, 1.0, vr1));
  }
  CView vr3{XP.p, V, VV, V, V, OVV, 1};
  ACES_TRY(G(o * v, o * v, o * v, 1.0, Tpp.p, OV, WB.p, OV, 1.0, vr3));
  // Z2 += XP + XP^T(ia<->jb) (SUMSYM / SUMRNG)
  ACES_TRY(perm(Z2.p, o, o, v, v, 1.0,
                {PT(XP.p, 1.0, st2[0], st2[1], st2[2], st2[3]),
                 PT(XP.p, 1.0, st2[1], st2[0], st2[3], st2[2])}));
  return ACES_OK;
}

// Particle-particle ladder Z2[ij,ab] += sum_cd <ab|cd> tau[ij,cd] on symmetric
// and antisymmetric pair combinations (the reference's RHF a<=b packing,
// vcc/ladab1.F:55-64 with SYMEXP4).  With <ba|dc> = <ab|cd>:
//   S[ij,a<=b] = sum_{c<=d} U+[ab,cd] tau+[ij,cd],  U+ = (<ab|cd> + <ab|dc>)/2 (c<d), <ab|cc>
//   A[ij,a<b]  = sum_{c<d}  U-[ab,cd] tau-[ij,cd],  U- = (<ab|cd> - <ab|dc>)/2
//   tau+ = tau[cd] + tau[dc] (c<d), tau[cc];  tau- = tau[cd] - tau[dc]
//   Z2[ab] += S + A,  Z2[ba] += S - A,  Z2[aa] += S
// Two contractions of (v(v+1)/2)^2 and (v(v-1)/2)^2 x o^2 instead of v^4 x o^2:
// half the flops.  U+/U- are built once from the dense <ab|cd> (or the list).
// The map is linear in tau and needs no symmetry of it, so the Lambda
// backward pass calls it with (Z2 adjoint, tau adjoint) for in and out.
int CCEngine::ladder_packed_blocks(const double *in, double *out) {
  const int nir = state().sym.nirrep;
  LadderBlocks &Lb = ladb;
  if (!Up.p) {
    // pair lists by pair irrep: symmetric c <= d and antisymmetric c < d (d
    // slowest), occupied pairs ij by irrep; local indices of every pair
    std::vector<int> pp, mm, pidx((size_t)v * v, -1), midx((size_t)v * v, -1), ijs, ijl(o * o);
    Lb.nirrep = nir;
    Lb.o = o;
    Lb.v = v;
    Lb.offP[0] = Lb.offM[0] = Lb.offIJ[0] = 0;
    for (int g = 0; g < nir; ++g) {
      int np_g = 0, nm_g = 0, nij = 0;
      for (int d = 0; d < v; ++d)
        for (int c = 0; c <= d; ++c) {
          if ((irr_v[c] ^ irr_v[d]) != g) continue;
          pp.push_back(c);
          pp.push_back(d);
          pidx[(size_t)c * v + d] = np_g++;
          if (c < d) {
            mm.push_back(c);
            mm.push_back(d);
            midx[(size_t)c * v + d] = nm_g++;
          }
        }
      for (int ij = 0; ij < o * o; ++ij)
        if ((irr_o[ij / o] ^ irr_o[ij % o]) == g) {
          ijs.push_back(ij);
          ijl[ij] = nij++;
        }
      Lb.nP[g] = np_g;
      Lb.nM[g] = nm_g;
      Lb.nIJ[g] = nij;
      Lb.offP[g + 1] = Lb.offP[g] + np_g;
      Lb.offM[g + 1] = Lb.offM[g] + nm_g;
      Lb.offIJ[g + 1] = Lb.offIJ[g] + nij;
    }
    for (int g = nir; g < 8; ++g) Lb.nP[g] = Lb.nM[g] = Lb.nIJ[g] = 0;
    Lb.offUp[0] = Lb.offUm[0] = 0;
    for (int g = 0; g < nir; ++g) {
      Lb.offUp[g + 1] = Lb.offUp[g] + (long long)Lb.nP[g] * Lb.nP[g];
      Lb.offUm[g + 1] = Lb.offUm[g] + (long long)Lb.nM[g] * Lb.nM[g];
    }
    std::vector<int> tab;
    auto put = [&](const std::vector<int> &x) {
      const size_t at = tab.size();
      tab.insert(tab.end(), x.begin(), x.end());
      return at;
    };
    std::vector<int> io(irr_o.begin(), irr_o.end()), iv(irr_v.begin(), irr_v.end());
    const size_t a_pp = put(pp), a_mm = put(mm), a_pi = put(pidx), a_mi = put(midx),
                 a_ijs = put(ijs), a_ijl = put(ijl), a_io = put(io), a_iv = put(iv);
    ACES_TRY(alloc(ladpairs, (tab.size() + 1) / 2 + 1));
    ACES_CUDA(cudaMemcpyAsync(ladpairs.p, tab.data(), tab.size() * sizeof(int),
                              cudaMemcpyHostToDevice, st));
    const int *base = reinterpret_cast<const int *>(ladpairs.p);
    Lb.pp = base + a_pp;
    Lb.mm = base + a_mm;
    Lb.pidx = base + a_pi;
    Lb.midx = base + a_mi;
    Lb.ijs = base + a_ijs;
    Lb.ijl = base + a_ijl;
    Lb.irr_o = base + a_io;
    Lb.irr_v = base + a_iv;
    ACES_TRY(alloc(Up, (size_t)std::max(1LL, Lb.offUp[nir])));
    ACES_TRY(alloc(Um, (size_t)std::max(1LL, Lb.offUm[nir])));
    launch_ladder_pack_v_blk(Up.p, Um.p, I_vvvv.p, Lb, st);
    ACES_CUDA(cudaStreamSynchronize(st));
  }
  // per-call blocks of the vector's symmetry
  Lb.hs = ladder_sym;
  Lb.offTp[0] = Lb.offTm[0] = 0;
  for (int g = 0; g < nir; ++g) {
    const long long rows = Lb.nIJ[g ^ Lb.hs];
    Lb.offTp[g + 1] = Lb.offTp[g] + rows * Lb.nP[g];
    Lb.offTm[g + 1] = Lb.offTm[g] + rows * Lb.nM[g];
  }
  ACES_TRY(alloc(taup, (size_t)std::max(1LL, Lb.offTp[nir])));
  ACES_TRY(alloc(taum, (size_t)std::max(1LL, Lb.offTm[nir])));
  ACES_TRY(alloc(Sld, (size_t)std::max(1LL, Lb.offTp[nir])));
  ACES_TRY(alloc(Ald, (size_t)std::max(1LL, Lb.offTm[nir])));
  memo_written(taup.p, std::max(1LL, Lb.offTp[nir]));
  memo_written(taum.p, std::max(1LL, Lb.offTm[nir]));
  launch_ladder_pack_tau_blk(taup.p, taum.p, in, Lb, st);
  // block products S_g = U+_g tau+_g^T, A_g = U-_g tau-_g^T, three per grouped launch
  std::vector<GArgs> probs;
  for (int g = 0; g < nir; ++g) {
    const int rows = Lb.nIJ[g ^ Lb.hs];
    if (rows == 0) continue;
    const int np_g = Lb.nP[g], nm_g = Lb.nM[g];
    if (np_g > 0)
      probs.push_back({np_g, rows, np_g, Up.p + Lb.offUp[g], np_g, taup.p + Lb.offTp[g], np_g,
                       cview_colmajor(Sld.p + Lb.offTp[g], np_g), true, false});
    if (nm_g > 0)
      probs.push_back({nm_g, rows, nm_g, Um.p + Lb.offUm[g], nm_g, taum.p + Lb.offTm[g], nm_g,
                       cview_colmajor(Ald.p + Lb.offTm[g], nm_g), true, false});
  }
  // the largest products first, so each grouped launch pairs similar sizes
  std::sort(probs.begin(), probs.end(), [](const GArgs &x, const GArgs &y) {
    return (double)x.M * x.N * x.K > (double)y.M * y.N * y.K;
  });
  for (size_t q = 0; q < probs.size(); q += 3)
    ACES_TRY(Ggroup(probs.data() + q, (int)std::min<size_t>(3, probs.size() - q), 0.0));
  memo_written(out, (long long)o * o * v * v);
  launch_ladder_unpack_blk(out, Sld.p, Ald.p, Lb, st);
  ACES_CUDA(cudaGetLastError());
  return ACES_OK;
}

int CCEngine::ladder_packed(const double *in, double *out) {
  if (state().sym.nirrep > 1) return ladder_packed_blocks(in, out);
  const int np = v * (v + 1) / 2, nm = v * (v - 1) / 2, oo = o * o;
  if (!Up.p) {
    // pair tables: p(c,d) = d(d+1)/2 + c (c <= d), m(c,d) = d(d-1)/2 + c (c < d)
    std::vector<int> pr((size_t)2 * (np + nm));
    for (int d = 0; d < v; ++d)
      for (int c = 0; c <= d; ++c) {
        const int p = d * (d + 1) / 2 + c;
        pr[2 * p] = c;
        pr[2 * p + 1] = d;
        if (c < d) {
          const int m = d * (d - 1) / 2 + c;
          pr[2 * (np + m)] = c;
          pr[2 * (np + m) + 1] = d;
        }
      }
    ACES_TRY(alloc(ladpairs, (pr.size() + 1) / 2));
    ACES_CUDA(cudaMemcpyAsync(ladpairs.p, pr.data(), pr.size() * sizeof(int),
                              cudaMemcpyHostToDevice, st));
    ACES_TRY(alloc(Up, (size_t)np * np));
    ACES_TRY(alloc(Um, (size_t)std::max(nm, 1) * std::max(nm, 1)));
    launch_ladder_pack_v(Up.p, Um.p, I_vvvv.p, (const int *)ladpairs.p, v, st);
    ACES_CUDA(cudaStreamSynchronize(st));
  }
  ACES_TRY(alloc(taup, (size_t)oo * np));
  ACES_TRY(alloc(taum, (size_t)oo * std::max(nm, 1)));
  ACES_TRY(alloc(Sld, (size_t)oo * np));
  ACES_TRY(alloc(Ald, (size_t)oo * std::max(nm, 1)));
  memo_written(taup.p, (long long)oo * np);
  memo_written(taum.p, (long long)oo * std::max(nm, 1));
  if (memo_on && nm > 0 && splits(np, oo, np) && splits(nm, oo, nm)) {
    // inside a residual pass whose grouped launch splits: tau+- straight
    // into the planes of its B operands, no FP64 copy
    MemoEntry *mp = nullptr, *mm = nullptr;
    ACES_TRY(memo_planes(taup.p, oo, np, &mp));
    ACES_TRY(memo_planes(taum.p, oo, nm, &mm));
    LadderPlanes pl;
    pl.hi_p = (__nv_bfloat16 *)mp->op.hi;
    pl.lo_p = (__nv_bfloat16 *)mp->op.lo;
    pl.hi_m = (__nv_bfloat16 *)mm->op.hi;
    pl.lo_m = (__nv_bfloat16 *)mm->op.lo;
    pl.kp_p = mp->op.k_pad;
    pl.kp_m = mm->op.k_pad;
    launch_ladder_pack_tau(taup.p, taum.p, in, v, oo, st, &pl);
    mp->valid = mm->valid = true;
    mp->fp64 = mm->fp64 = false;
  } else {
    launch_ladder_pack_tau(taup.p, taum.p, in, v, oo, st);
  }
  // both products in one grouped launch (their tiles fill each other's last wave)
  const GArgs g[2] = {{np, oo, np, Up.p, np, taup.p, np, cview_colmajor(Sld.p, np), true, false},
                      {nm, oo, nm, Um.p, nm, taum.p, nm, cview_colmajor(Ald.p, nm), true, false}};
  ACES_TRY(Ggroup(g, nm > 0 ? 2 : 1, 0.0));
  memo_written(out, (long long)o * o * v * v);
  launch_ladder_unpack(out, Sld.p, Ald.p, v, oo, st);
  ACES_CUDA(cudaGetLastError());
  return ACES_OK;
}

// The residual pass, directly or through its captured graph.  The first pass
// allocates (intermediates, split caches, packed ladder); the second is
// captured with every buffer in place, so the graph's kernels keep reading and
// writing the same addresses on every replay.
int CCEngine::residual_run() {
  if (!use_graph || recording) return residual();
  if (residual_exec) {
    ACES_CUDA(cudaGraphLaunch(residual_exec, st));
    g_launches.fetch_add(residual_launches, std::memory_order_relaxed);
    gemm_flops += residual_flops;
    return ACES_OK;
  }
  if (residual_passes++ == 0) return residual();  // first pass: allocations happen here
  const long long l0 = g_launches.load();
  const double f0 = gemm_flops;
  cudaGraph_t graph = nullptr;
  ACES_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  capturing = true;
  const int s = residual();
  capturing = false;
  const cudaError_t ce = cudaStreamEndCapture(st, &graph);
  if (s != ACES_OK) {
    if (graph) cudaGraphDestroy(graph);
    return s;
  }
  if (ce != cudaSuccess) {
    set_error("residual graph capture failed: %s", cudaGetErrorString(ce));
    return ACES_ERR_CUDA;
  }
  residual_launches = g_launches.load() - l0;
  residual_flops = gemm_flops - f0;
  const cudaError_t ie = cudaGraphInstantiate(&residual_exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) {
    residual_exec = nullptr;
    set_error("residual graph instantiation failed: %s", cudaGetErrorString(ie));
    return ACES_ERR_CUDA;
  }
  ACES_CUDA(cudaGraphLaunch(residual_exec, st));
  return ACES_OK;
}

// One CC cycle: residual, Jacobi update, energy, DIIS (vcc/vcc.F:797-1087).
int CCEngine::iteration(int icycle, int exporder, double *e3, double *res, double *dres,
                        bool *extrap, bool lambda) {
  const long long len = (long long)o * v + (long long)o * o * v * v;
  const long long ov = (long long)o * v;
  double *d = dev_small.p;  // [0..2] energy, [3] res, [4] dres, [8..32] dots, [40..64] coef
  double *cur = lambda ? L.p : X.p;
  double *nxt = lambda ? Ln.p : Xn.p;
  if (!lambda) {
    ACES_TRY(residual_run());
    launch_newt(t2n(), Z2.p, t1n(), Z1.p, eo.p, ev.p, o, v, st);
    // DAMP_CC_RESIDUAL after NEWT2 (vcc/vcc.F:1031-1033); the energy, the
    // error vector and the next iterate are those of the damped amplitudes
    if (damp != 1.0) launch_blend(Xn.p, X.p, damp, len, st);
    launch_energy(d, t2n(), t1n(), I_oovv.p, fov.p, o, v, scratch.p, st);
  } else {
    // Lambda: new multipliers = (dE/dT + (dZ/dT)^T lambda) / D
    ACES_TRY(lambda_rhs());
    launch_newt(Ln.p + ov, lrhs.p + ov, Ln.p, lrhs.p, eo.p, ev.p, o, v, st);
    ACES_CUDA(cudaMemsetAsync(d, 0, 3 * sizeof(double), st));
  }
  int ndimr = icycle < exporder ? icycle : exporder;
  int idimr = (icycle - 1) % exporder;
  if ((int)hx.size() < exporder) {
    hx.resize(exporder);
    he.resize(exporder);
  }
  // every history slot is allocated on the first cycle, so no later (timed)
  // cycle waits on the allocator
  for (int k = 0; k < exporder; ++k)
    if (!hx[k].p) {
      ACES_TRY(alloc(hx[k], len));
      ACES_TRY(alloc(he[k], len));
    }
  ACES_TRY(copy(hx[idimr].p, cur, len));
  std::vector<const double *> hp(ndimr);
  for (int k = 0; k < ndimr; ++k) hp[k] = he[k].p;
  // error vector, its largest element and its DIIS dots in one pass
  ACES_TRY(launch_diff_stats(he[idimr].p, nxt, cur, hp.data(), ndimr, idimr, o, v, scratch.p,
                             d + 3, d + 8, st));
  double hd[40];
  ACES_CUDA(cudaMemcpyAsync(hd, d, 40 * 8, cudaMemcpyDeviceToHost, st));
  ACES_CUDA(cudaStreamSynchronize(st));
  if (int tcs = tc_status_and_clear()) {
    set_error("tensor-core contraction gave up waiting (code %d) at cycle %d", tcs, icycle);
    return ACES_ERR_TIMEOUT;
  }
  e3[0] = hd[1];  // E_AA (printed alpha-alpha part)
  e3[1] = hd[0];  // E_AB
  e3[2] = 2.0 * hd[1] + hd[0] + hd[2];
  // convergence on the undamped difference (vcc/dodiis0.F:93-97)
  *res = (!lambda && damp != 1.0) ? hd[3] / damp : hd[3];
  if (Bh.size() != 625) Bh.assign(625, 0.0);
  for (int k = 0; k < ndimr; ++k) {
    Bh[k * 25 + idimr] = hd[8 + k];
    Bh[idimr * 25 + k] = hd[8 + k];
  }
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(e3[k])) {
      set_error("non-finite CC energy at cycle %d", icycle);
      return ACES_ERR_NAN;
    }
  ACES_CUDA(cudaMemcpyAsync(Bmat.p, Bh.data(), 625 * 8, cudaMemcpyHostToDevice, st));
  int *status = reinterpret_cast<int *>(d + 36);
  launch_diis_solve(d + 40, status, Bmat.p, ndimr, st);
  // DIIS residual dvec = sum_i c_i e_i (vcc/dodiis0.F:131-146)
  std::vector<const double *> pe(ndimr);
  for (int k = 0; k < ndimr; ++k) pe[k] = he[k].p;
  ACES_TRY(alloc(dvec, len));
  launch_lincomb_absmax(dvec.p, d + 40, pe.data(), ndimr, o, v, scratch.p, d + 4, st);
  int hstat = 0;
  ACES_CUDA(cudaMemcpyAsync(&hstat, status, 4, cudaMemcpyDeviceToHost, st));
  ACES_CUDA(cudaMemcpyAsync(dres, d + 4, 8, cudaMemcpyDeviceToHost, st));
  ACES_CUDA(cudaStreamSynchronize(st));
  if (hstat) {
    set_error("DIIS bordered system singular at cycle %d", icycle);
    return ACES_ERR_SINGULAR;
  }
  *extrap = ndimr >= 2;
  return ACES_OK;
}

// accept the new amplitudes: extrapolated (DIIS) or plain Jacobi (DRMOVE)
int accept_update(CCEngine &E, bool extrap, int ndimr, bool lambda) {
  const long long len = (long long)E.o * E.v + (long long)E.o * E.o * E.v * E.v;
  double *cur = lambda ? E.L.p : E.X.p;
  double *nxt = lambda ? E.Ln.p : E.Xn.p;
  if (extrap) {
    std::vector<const double *> px(ndimr);
    for (int k = 0; k < ndimr; ++k) px[k] = E.hx[k].p;
    launch_lincomb(cur, E.dvec.p, E.dev_small.p + 40, px.data(), ndimr, len, E.st);
  } else {
    ACES_TRY(E.copy(cur, nxt, len));
  }
  ACES_CUDA(cudaGetLastError());
  return ACES_OK;
}

int CCEngine::write_amplitudes(const double *a1, const double *a2, int list1, int list2ab,
                               int list2aa) {
  const long long O = o, V = v;
  const SymInfo &s = state().sym;
  // doubles (AB) -> list2ab (13,14): dense [a,b,i,j] = a2[i,j,a,b]
  DBuf tmpb;
  ACES_TRY(alloc(tmpb, O * O * V * V));
  const long long st2[4] = {O * V * V, V * V, V, 1};
  ACES_TRY(perm(tmpb.p, v, v, o, o, 0.0, {PT(a2, 1.0, st2[2], st2[3], st2[0], st2[1])}));
  {
    DevMap dm;
    ACES_TRY(make_map(dm, list2ab, 13, 14, irr_o, irr_v, true));
    launch_scatter(tmpb.p, dm.m, st);
    ACES_CUDA(cudaStreamSynchronize(st));
  }
  // same-spin doubles -> list2aa (1,3): dense [a,b,i,j] = a2[i,j,a,b] - a2[i,j,b,a]
  ACES_TRY(perm(tmpb.p, v, v, o, o, 0.0,
                {PT(a2, 1.0, st2[2], st2[3], st2[0], st2[1]),
                 PT(a2, -1.0, st2[3], st2[2], st2[0], st2[1])}));
  {
    DevMap dm;
    ACES_TRY(make_map(dm, list2aa, 1, 3, irr_o, irr_v, true));
    launch_scatter(tmpb.p, dm.m, st);
    ACES_CUDA(cudaStreamSynchronize(st));
  }
  // singles -> list1 irrep 1, one column over (a,i) pairs of type 9
  {
    int n9 = s.irpdpd[0][8];
    ACES_TRY(aces_list_touch(1, n9, 1, list1, 0));
    std::vector<double> h1((size_t)o * v), col((size_t)n9, 0.0);
    ACES_CUDA(cudaMemcpy(h1.data(), a1, h1.size() * 8, cudaMemcpyDeviceToHost));
    std::vector<int> lo(o), lv(v);
    int cnt[8] = {0};
    for (int i = 0; i < o; ++i) lo[i] = cnt[irr_o[i]]++;
    for (int k = 0; k < 8; ++k) cnt[k] = 0;
    for (int a = 0; a < v; ++a) lv[a] = cnt[irr_v[a]]++;
    for (int i = 0; i < o; ++i)
      for (int a = 0; a < v; ++a)
        if (irr_o[i] == irr_v[a])
          col[pair_index(s, 9, irr_v[a], lv[a], irr_o[i], lo[i])] = h1[(size_t)i * v + a];
    ACES_TRY(aces_putlst(col.data(), 1, 1, 1, list1));
  }
  dev_free(tmpb.p);
  return ACES_OK;
}

// T1 -> list 90, T2(AB) -> list 46, T2(AA) -> list 44 (vcc/vcc.F list map)
int CCEngine::write_back() { return write_amplitudes(t1(), t2(), 90, 46, 44); }

static CCEngine *g_engine = nullptr;
CCEngine *engine_instance(bool create) {
  if (!g_engine && create) g_engine = new CCEngine();
  return g_engine;
}
void engine_reset() {
  delete g_engine;
  g_engine = nullptr;
}

}  // namespace acesb200

using namespace acesb200;

extern "C" int xvcc_run(aces_cc_config *cfg) {
  if (!cfg) return ACES_ERR_ARG;
  State &stt = state();
  std::lock_guard<std::recursive_mutex> lk(stt.mu);
  if (cfg->cc_exporder < 1 || cfg->cc_exporder > 25 || cfg->cc_maxcyc < 1) {
    set_error("xvcc_run: cc_exporder must be 1..25 and cc_maxcyc >= 1");
    return ACES_ERR_ARG;
  }
  if (cfg->precision != ACES_PREC_FP64 && cfg->precision != ACES_PREC_BF16X3) return ACES_ERR_ARG;
  engine_reset();
  CCEngine &E = *engine_instance(true);
  E.prec = cfg->precision;
  E.use_graph = cfg->use_graph != 0;
  if (!(cfg->damp >= 0.0 && cfg->damp <= 1.0)) {
    set_error("xvcc_run: damp %g outside [0, 1] (0 means no damping)", cfg->damp);
    return ACES_ERR_ARG;
  }
  E.damp = cfg->damp == 0.0 ? 1.0 : cfg->damp;
  cudaEvent_t ev0, ev1;
  ACES_CUDA(cudaEventCreate(&ev0));
  ACES_CUDA(cudaEventCreate(&ev1));
  {
    auto t0 = std::chrono::steady_clock::now();
    ACES_TRY(E.load_from_lists());
    ACES_TRY(E.setup_intermediates());
    bool read = false;
    if (cfg->tguess) ACES_TRY(E.read_guess(&read));
    if (!read) ACES_TRY(E.mp2_guess());
    cfg->tguess = read ? 1 : 0;
    ACES_CUDA(cudaStreamSynchronize(E.st));
    cfg->seconds_setup =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  const double tol = std::pow(10.0, -cfg->cc_conv);
  float ms_lad_total = 0.f;
  int ntimed = 0;
  long long launches_timed = 0;
  double e3[3] = {0, 0, 0}, res = 0, dres = 0;
  bool converged = false;
  int icycle = 0;
  float ms_total = 0.f;
  for (icycle = 1; icycle <= cfg->cc_maxcyc; ++icycle) {
    bool extrap = false;
    long long l0 = g_launches.load();
    E.gemm_flops = 0.0;
    ACES_CUDA(cudaEventRecord(ev0, E.st));
    ACES_TRY(E.iteration(icycle, cfg->cc_exporder, e3, &res, &dres, &extrap));
    cfg->flops_per_iter = E.gemm_flops;
    int ndimr = icycle < cfg->cc_exporder ? icycle : cfg->cc_exporder;
    bool conv = std::fabs(res) < tol;
    if (!conv) ACES_TRY(accept_update(E, extrap, ndimr, false));
    ACES_CUDA(cudaEventRecord(ev1, E.st));
    ACES_CUDA(cudaEventSynchronize(ev1));
    float ms = 0.f, msl = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    if (cudaEventElapsedTime(&msl, E.ev_lad0, E.ev_lad1) != cudaSuccess) {
      cudaGetLastError();
      msl = 0.f;
    }
    if (icycle > cfg->timing_warmup) {
      ms_total += ms;
      ms_lad_total += msl;
      ntimed++;
      launches_timed += g_launches.load() - l0;
    }
    if (cfg->verbose)
      printf("  cycle %3d  E(corr) = %.12f  max res = % .8e  max DIIS res = % .8e  %.3f ms\n",
             icycle, e3[2], res, dres, ms);
    if (conv) {
      converged = true;
      break;
    }
  }
  if (icycle > cfg->cc_maxcyc) icycle = cfg->cc_maxcyc;
  // final energy of the accepted amplitudes (vcc/vcc.F:1101)
  double *d = E.dev_small.p;
  launch_energy(d, E.t2(), E.t1(), E.I_oovv.p, E.fov.p, E.o, E.v, E.scratch.p, E.st);
  double hd[3];
  ACES_CUDA(cudaMemcpyAsync(hd, d, 24, cudaMemcpyDeviceToHost, E.st));
  ACES_CUDA(cudaStreamSynchronize(E.st));
  cfg->e_ccsd = 2.0 * hd[1] + hd[0] + hd[2];
  cfg->last_residual = res;
  cfg->ncycle = icycle;
  cfg->converged = converged ? 1 : 0;
  cfg->seconds_per_iter = ntimed ? ms_total * 1e-3 / ntimed : 0.0;
  cfg->seconds_ladder = ntimed ? ms_lad_total * 1e-3 / ntimed : 0.0;
  cfg->launches_per_iter = ntimed ? launches_timed / ntimed : 0;
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  ACES_TRY(E.write_back());
  aces_putrec("CCSDENRG", 8, &cfg->e_ccsd);
  E.have_amplitudes = converged;
  E.have_lambda = false;
  if (!converged) {
    set_error("CC equations did not converge in %d cycles", cfg->cc_maxcyc);
    return ACES_ERR_NOCONV;
  }
  if (cfg->triples) {
    // (T) on the converged amplitudes (vcc/vcc.F:1215 -> trp/trps.F)
    const int nr = cfg->triples_nranks > 0 ? cfg->triples_nranks : 1;
    if (cfg->triples_rank < 0 || cfg->triples_rank >= nr) {
      set_error("xvcc_run: triples_rank %d outside 0..%d", cfg->triples_rank, nr - 1);
      return ACES_ERR_ARG;
    }
    ACES_TRY(E.triples(&cfg->e_t4, &cfg->e_st5, &cfg->seconds_triples, cfg->triples_rank, nr));
    aces_putrec("E4T", 8, &cfg->e_t4);
    aces_putrec("E5ST", 8, &cfg->e_st5);
  }
  return ACES_OK;
}
