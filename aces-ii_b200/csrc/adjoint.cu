// adjoint.cu -- backward kernels and the reverse replay of a recorded residual.
#include <algorithm>

#include "adjoint.cuh"
#include "engine.cuh"
#include "perm_plan.cuh"

namespace acesb200 {

namespace {
__device__ __forceinline__ long long view_off(const CView &C, long long m, long long n) {
  return cview_off(C, (int)m, (int)n);
}

__global__ void k_view_gather(double *__restrict__ dense, CView C, int M, int N, double scale) {
  long long total = (long long)M * N;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    long long m = idx / N, n = idx % N;
    dense[idx] = scale * C.p[view_off(C, m, n)];
  }
}

__global__ void k_view_scale(CView C, int M, int N, double value) {
  long long total = (long long)M * N;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    long long m = idx / N, n = idx % N;
    double *p = C.p + view_off(C, m, n);
    *p = value == 0.0 ? 0.0 : value * *p;
  }
}

__global__ void k_perm_scatter_add(double *__restrict__ src_bar, const double *__restrict__ out_bar,
                                   double alpha, long long s0, long long s1, long long s2,
                                   long long s3, int n0, int n1, int n2, int n3) {
  long long total = (long long)n0 * n1 * n2 * n3;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    long long r = idx;
    int i3 = r % n3; r /= n3;
    int i2 = r % n2; r /= n2;
    int i1 = r % n1; r /= n1;
    int i0 = (int)r;
    // a permutation is injective: no two threads update the same element
    src_bar[i0 * s0 + i1 * s1 + i2 * s2 + i3 * s3] += alpha * out_bar[idx];
  }
}

__global__ void k_axpy(double *__restrict__ y, const double *__restrict__ x, double a, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] += a * x[i];
}

__global__ void k_scale(double *__restrict__ y, double a, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = a == 0.0 ? 0.0 : a * y[i];
}

// t1_bar[i,a] += c * sum_jb taub[i,j,a,b] t1[j,b] + c * sum_jb taub[j,i,b,a] t1[j,b]
// one block per (i,a)
__global__ void k_tau_adj_t1(double *__restrict__ t1_bar, const double *__restrict__ taub,
                             const double *__restrict__ t1, double c, int o, int v) {
  int ia = blockIdx.x;
  int i = ia / v, a = ia % v;
  double s = 0.0;
  for (int jb = threadIdx.x; jb < o * v; jb += blockDim.x) {
    int j = jb / v, b = jb % v;
    s += taub[(((long long)i * o + j) * v + a) * v + b] * t1[jb];
    s += taub[(((long long)j * o + i) * v + b) * v + a] * t1[jb];
  }
  __shared__ double sh[8];
  for (int off = 16; off; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    t1_bar[ia] += c * t;
  }
}

unsigned blocks_for(long long n) {
  long long nb = (n + 255) / 256;
  if (nb > 148 * 32) nb = 148 * 32;
  if (nb < 1) nb = 1;
  return (unsigned)nb;
}
}  // namespace

void launch_view_gather(double *dense, const CView &C, int M, int N, double scale,
                        cudaStream_t st) {
  k_view_gather<<<blocks_for((long long)M * N), 256, 0, st>>>(dense, C, M, N, scale);
  count_launch();
}
void launch_view_scale(const CView &C, int M, int N, double value, cudaStream_t st) {
  k_view_scale<<<blocks_for((long long)M * N), 256, 0, st>>>(C, M, N, value);
  count_launch();
}
void launch_perm_scatter_add(double *src_bar, const double *out_bar, const PermTerm &t,
                             const int n[4], cudaStream_t st) {
  long long total = (long long)n[0] * n[1] * n[2] * n[3];
  k_perm_scatter_add<<<blocks_for(total), 256, 0, st>>>(src_bar, out_bar, t.alpha, t.s[0], t.s[1],
                                                        t.s[2], t.s[3], n[0], n[1], n[2], n[3]);
  count_launch();
}
void launch_axpy(double *y, const double *x, double a, long long n, cudaStream_t st) {
  k_axpy<<<blocks_for(n), 256, 0, st>>>(y, x, a, n);
  count_launch();
}
void launch_scale(double *y, double a, long long n, cudaStream_t st) {
  k_scale<<<blocks_for(n), 256, 0, st>>>(y, a, n);
  count_launch();
}
void launch_tau_adjoint(double *t2_bar, double *t1_bar, const double *tau_bar, const double *t1,
                        double c, int o, int v, cudaStream_t st) {
  long long n = (long long)o * o * v * v;
  if (t2_bar) launch_axpy(t2_bar, tau_bar, 1.0, n, st);
  if (t1_bar) {
    k_tau_adj_t1<<<o * v, 256, 0, st>>>(t1_bar, tau_bar, t1, c, o, v);
    count_launch();
  }
}

// ---------------------------------------------------------------------------
// engine side: buffer registry, activity, tape recording and reverse replay
// ---------------------------------------------------------------------------
DBuf *CCEngine::owner(const void *p) {
  const char *q = (const char *)p;
  for (DBuf *b : registry())
    if (b->p && q >= (const char *)b->p && q < (const char *)(b->p + b->n)) return b;
  for (auto &b : hx) if (b.p && q >= (const char *)b.p && q < (const char *)(b.p + b.n)) return &b;
  for (auto &b : he) if (b.p && q >= (const char *)b.p && q < (const char *)(b.p + b.n)) return &b;
  return nullptr;
}

bool CCEngine::is_active(const void *p) {
  DBuf *b = owner(p);
  if (!b) return false;
  for (DBuf *a : active)
    if (a == b) return true;
  return false;
}

void CCEngine::mark_active(const void *p) {
  DBuf *b = owner(p);
  if (!b || is_active(p)) return;
  active.push_back(b);
}

double *CCEngine::adj(const void *p) {
  DBuf *b = owner(p);
  if (!b) return nullptr;
  auto it = adjoint.find(b);
  if (it == adjoint.end()) {
    DBuf a;
    if (alloc(a, b->n) != ACES_OK) return nullptr;
    it = adjoint.emplace(b, a).first;
  }
  return it->second.p + ((const double *)p - b->p);
}

int CCEngine::tmp(DBuf &b, size_t n) { return alloc(b, n); }

// transpose of a constant operand (rows x cols, leading dim ld) -> [cols, rows]
const double *CCEngine::transposed(const double *src, int rows, int cols, long long ld, bool cst,
                                   DBuf &scratch) {
  if (cst && rows == cols && ld == cols)
    for (const double *sp : symmetric)
      if (sp == src) return src;
  const auto key = std::make_tuple(src, rows, cols, ld);
  if (cst) {
    auto it = tcache.find(key);
    if (it != tcache.end()) return it->second.p;
  }
  DBuf *dst = &scratch;
  DBuf fresh;
  if (cst) dst = &fresh;
  if (alloc(*dst, (size_t)rows * cols) != ACES_OK) return nullptr;
  PermSpec s;
  s.n[0] = 1; s.n[1] = 1; s.n[2] = cols; s.n[3] = rows;
  s.nterms = 1;
  s.beta = 0.0;
  s.t[0].src = src;
  s.t[0].alpha = 1.0;
  s.t[0].s[0] = 0; s.t[0].s[1] = 0; s.t[0].s[2] = 1; s.t[0].s[3] = ld;
  if (permute(dst->p, s, st) != ACES_OK) return nullptr;
  if (cst) {
    tcache[key] = fresh;
    return fresh.p;
  }
  return dst->p;
}

const double *CCEngine::tape_transposed(const double *src, int rows, int cols, long long ld) {
  const auto key = std::make_tuple(src, rows, cols, ld);
  auto it = tape_tcache.find(key);
  if (it != tape_tcache.end()) return it->second.p;
  DBuf fresh;
  if (alloc(fresh, (size_t)rows * cols) != ACES_OK) return nullptr;
  PermSpec s;
  s.n[0] = 1; s.n[1] = 1; s.n[2] = cols; s.n[3] = rows;
  s.nterms = 1;
  s.beta = 0.0;
  s.t[0].src = src;
  s.t[0].alpha = 1.0;
  s.t[0].s[0] = 0; s.t[0].s[1] = 0; s.t[0].s[2] = 1; s.t[0].s[3] = ld;
  if (permute(fresh.p, s, st) != ACES_OK) {
    dev_free(fresh.p);
    return nullptr;
  }
  tape_tcache[key] = fresh;
  return fresh.p;
}

void CCEngine::tape_cache_clear() {
  for (auto &kv : tape_tcache) {
    const double *p = kv.second.p;
    for (auto e = split_cache.begin(); e != split_cache.end();) {
      if (e->src == p) {
        if (e->op.hi) dev_free(e->op.hi);
        e = split_cache.erase(e);
      } else {
        ++e;
      }
    }
    if (kv.second.p) dev_free(kv.second.p);
  }
  tape_tcache.clear();
}

int CCEngine::backward() {
  // walk the tape in reverse; adjoint buffers already hold the seeds
  const bool rec = recording;
  recording = false;
  for (auto it = tape.rbegin(); it != tape.rend(); ++it) {
    TapeOp &op = *it;
    if (op.kind == TapeOp::GEMM) {
      double *cbar_base = adj(op.C.p);
      if (!cbar_base) return ACES_ERR_NOMEM;
      CView cb = op.C;
      cb.p = cbar_base;
      if (op.a_act || op.b_act) {
        // C_bar as an M x N row-major matrix (Cm, ldcm) and/or its transpose
        // (Ct, ldct): a plain row- or column-major output view is read in
        // place, any other view is gathered first; alpha goes to the products
        const bool plain = cb.mdiv > 0x7fffffff && cb.ndiv > 0x7fffffff;
        const double *Cm = nullptr, *Ct = nullptr;
        long long ldcm = 0, ldct = 0;
        if (plain && cb.sn0 == 1 && cb.sm0 >= op.N) {
          Cm = cbar_base;
          ldcm = cb.sm0;
        } else if (plain && cb.sm0 == 1 && cb.sn0 >= op.M) {
          Ct = cbar_base;
          ldct = cb.sn0;
        } else {
          ACES_TRY(tmp(bwdC, (size_t)op.M * op.N));
          launch_view_gather(bwdC.p, cb, op.M, op.N, 1.0, st);
          Cm = bwdC.p;
          ldcm = op.N;
        }
        // the forward operands are fixed for the tape's life (constants, or
        // values recorded at the converged amplitudes): their transposes are
        // cached, so are their splits
        if (op.a_act) {
          // A_bar[m,k] += alpha sum_n C_bar[m,n] B[n,k]
          const double *Bt = op.b_act ? tape_transposed(op.B, op.N, op.K, op.ldb)
                                      : transposed(op.B, op.N, op.K, op.ldb, true, bwdB);
          if (!Bt) return ACES_ERR_NOMEM;
          const double *A_ = Cm;
          long long lda_ = ldcm;
          if (!A_) {
            A_ = transposed(Ct, op.N, op.M, ldct, false, bwdC);
            lda_ = op.N;
          }
          if (!A_) return ACES_ERR_NOMEM;
          ACES_TRY(G(op.M, op.K, op.N, op.alpha, A_, lda_, Bt, op.N, 1.0,
                     cview_rowmajor(adj(op.A), op.lda), false, true));
        }
        if (op.b_act) {
          // B_bar[n,k] += alpha sum_m C_bar[m,n] A[m,k]
          const double *T_ = Ct;
          long long ldt_ = ldct;
          if (!T_) {
            T_ = transposed(Cm, op.M, op.N, ldcm, false, bwdD);
            ldt_ = op.M;
          }
          const double *At = op.a_act ? tape_transposed(op.A, op.M, op.K, op.lda)
                                      : transposed(op.A, op.M, op.K, op.lda, true, bwdA);
          if (!T_ || !At) return ACES_ERR_NOMEM;
          ACES_TRY(G(op.N, op.K, op.M, op.alpha, T_, ldt_, At, op.M, 1.0,
                     cview_rowmajor(adj(op.B), op.ldb), false, true));
        }
      }
      if (op.beta == 0.0)
        launch_view_scale(cb, op.M, op.N, 0.0, st);
      else if (op.beta != 1.0)
        launch_view_scale(cb, op.M, op.N, op.beta, st);
    } else if (op.kind == TapeOp::PERM) {
      double *obar = adj(op.out);
      if (!obar) return ACES_ERR_NOMEM;
      for (int t = 0; t < op.spec.nterms; ++t) {
        if (!op.t_act[t]) continue;
        const PermTerm &pt = op.spec.t[t];
        double *sbar = adj(pt.src);
        if (!sbar) return ACES_ERR_NOMEM;
        int m[4];
        long long ts[4];
        if (inverse_perm_plan(op.spec.n, pt.s, m, ts)) {
          // a dense bijection: the inverse resort, accumulated (beta = 1)
          ACES_TRY(perm(sbar, m[0], m[1], m[2], m[3], 1.0,
                        {PermTerm{obar, pt.alpha, {ts[0], ts[1], ts[2], ts[3]}}}));
        } else {
          launch_perm_scatter_add(sbar, obar, pt, op.spec.n, st);
        }
      }
      long long total = (long long)op.spec.n[0] * op.spec.n[1] * op.spec.n[2] * op.spec.n[3];
      if (op.spec.beta != 1.0) launch_scale(obar, op.spec.beta, total, st);
    } else if (op.kind == TapeOp::COPY) {
      double *dbar = adj(op.dst);
      if (is_active(op.src)) launch_axpy(adj(op.src), dbar, 1.0, (long long)op.count, st);
      launch_scale(dbar, 0.0, (long long)op.count, st);
    } else if (op.kind == TapeOp::LADDER) {
      // out += V in with V = <ab|cd> symmetric: in_bar += V out_bar, the same
      // packed ladder (out_bar is not changed: the forward accumulates)
      if (is_active(op.src)) {
        double *ob = adj(op.dst), *ib = adj(op.src);
        if (!ob || !ib) return ACES_ERR_NOMEM;
        ACES_TRY(ladder_packed(ob, ib));
      }
    } else if (op.kind == TapeOp::TAU) {
      double *tb = adj(op.tau);
      launch_tau_adjoint(adj(op.t2), adj(op.t1), tb, op.t1, op.c, o, v, st);
      launch_scale(tb, 0.0, (long long)o * o * v * v, st);
    }
    ACES_CUDA(cudaGetLastError());
  }
  recording = rec;
  return ACES_OK;
}

void CCEngine::zero_adjoints() {
  for (auto &kv : adjoint)
    if (kv.second.p) cudaMemsetAsync(kv.second.p, 0, kv.second.n * 8, st);
}

}  // namespace acesb200
