// engine.cuh -- the closed-shell CC engine shared by xvcc_run, xlambda_run and
// xdens_1pdm.
#pragma once
#include <cuda_runtime.h>

#include <deque>
#include <map>
#include <tuple>
#include <vector>

#include "adjoint.cuh"
#include "common.cuh"
#include "gemm.cuh"
#include "kernels.cuh"

namespace acesb200 {

// Dense FP64 device buffer owned by the engine.
struct DBuf {
  double *p = nullptr;
  size_t n = 0;
  bool borrowed = false;  // memory owned by the list store, never freed here
};

class CCEngine {
 public:
  int o = 0, v = 0, nmo = 0;
  int prec = ACES_PREC_FP64;
  // DAMP_CC (vcc/vcc.F:71): new amplitudes T_old + damp (T_new - T_old)
  double damp = 1.0;
  cudaStream_t st = 0;
  bool nonhf = false;
  // residual pass captured in a CUDA graph (use_graph): captured on the second
  // cycle, when every buffer it touches exists, and replayed afterwards
  bool use_graph = false;
  cudaGraphExec_t residual_exec = nullptr;
  long long residual_launches = 0;
  double residual_flops = 0.0;
  int residual_passes = 0;
  bool capturing = false;  // the residual pass is being captured into a graph
  int residual_run();

  // orbital data
  std::vector<double> eps_h;       // nmo, DPD order
  std::vector<int> irr_o, irr_v;   // orbital irreps
  DBuf eo, ev, foo, fvv, fov, offo, offv, fovT;

  // integrals (dense, physicists' notation)
  DBuf I_oooo, I_ooov, I_oovv, I_ovov, I_ovvv, I_vvvv;
  // precomputed resorted integrals
  DBuf L_oovv, LF, LovP, LooP, LmeP, I1, I2, IvP, IvP2, IX, IX2, WA0, WB0, IoP3, IvT,
      IooT, LT1;
  DBuf Ic, I1n;  // I1 - I2/2 and -I1 (the W(mbej) ring intermediates' integrals)

  // amplitudes: X = [t1 | t2] contiguous
  DBuf X, Xn, Z1, Z2;
  double *t1() { return X.p; }
  double *t2() { return X.p + (size_t)o * v; }
  double *t1n() { return Xn.p; }
  double *t2n() { return Xn.p + (size_t)o * v; }

  // temporaries
  DBuf tau, taut, tautP, tauT, U, Tp, Tpp, uT, wP, t2P, Y1, Y2, XnP, WA, WB, ZT, XP, Xmn, Wmnij,
      WmnT, t1T, Fae, Fmi, Fme, Fp, Fpp, FmiT, FppT, FmeT, tmp4;
  // packed particle-particle ladder (symmetric / antisymmetric pair combinations)
  DBuf Up, Um, taup, taum, Sld, Ald, ladpairs;
  // out[ij,ab] += <ab|cd> in[ij,cd] at half the dense flops
  int ladder_packed(const double *in, double *out);
  // the same on irrep blocks (more than one irrep): pair irrep g of (a,b) and
  // (c,d) with occupied pairs of irrep g ^ ladder_sym (0 for the amplitudes
  // and Lambda, the state's irrep for EOM products)
  int ladder_packed_blocks(const double *in, double *out);
  int ladder_sym = 0;
  LadderBlocks ladb{};  // block tables (device pointers into ladpairs)
  DBuf scratch, dev_small;  // reductions / DIIS scalars
  // DIIS history
  std::vector<DBuf> hx, he;
  DBuf Bmat;  // 25x25 on device
  DBuf dvec;  // DIIS residual sum_i c_i e_i
  std::vector<double> Bh;  // host copy (kept like /diisdat1/ in vcc/dodiis0.F)

  // split-precision operand cache (constant integrals)
  struct SplitEntry { const double *src; SplitOperand op; };
  std::deque<SplitEntry> split_cache;  // a deque: entries keep their address
  SplitOperand split_tmpA, split_tmpB, split_tmpG[6];
  // split operand of src (rows x K, leading dimension ld): cached when cst
  int split_get(const double *src, long long ld, int rows, int K, bool cst, SplitOperand &tmp,
                const SplitOperand **out);
  // Split planes of non-constant operands within one residual pass (memo_on):
  // the resorted amplitudes that permute_split writes straight into planes,
  // and every operand split once and read again by a later contraction of the
  // pass.  An entry stays valid until its source range is written again (the
  // engine's writers report every write through memo_written); fp64 = false
  // marks planes whose FP64 source was never written.  Entries keep their
  // planes (and addresses) across passes, so a captured residual graph
  // replays the same buffers.
  struct MemoEntry {
    const double *src;
    long long ld;
    int rows, K;
    bool valid, fp64;
    SplitOperand op;
  };
  std::deque<MemoEntry> memo;
  bool memo_on = false;
  MemoEntry &memo_slot(const double *src, long long ld, int rows, int K);
  // the entry of key as a rows x K operand (ld = K) with planes allocated
  int memo_planes(const double *key, int rows, int K, MemoEntry **out);
  void memo_written(const void *p, long long n);
  void memo_written(const CView &C, int M, int N);
  bool fp64_missing(const double *p) const;
  // the dispatch rule of G: does an M x N x K contraction take the split path
  bool splits(int M, int N, long long K) const;
  // perm (beta = 0) whose output is one contraction operand of rows x K
  // (K-contiguous): with memo_on and a consumer that splits, the planes are
  // written by the resort itself, plus the FP64 output only when keep_fp64
  int perm_split(double *out, int rows, int K, bool consumer_splits, bool keep_fp64, int n0,
                 int n1, int n2, int n3, std::initializer_list<PermTerm> terms);
  // several contractions C_g = A_g B_g^T + beta C_g in one grouped tensor-core
  // launch when all take the split path (else one G call each)
  struct GArgs {
    int M, N, K;
    const double *A;
    long long lda;
    const double *B;
    long long ldb;
    CView C;
    bool constA, constB;
  };
  int Ggroup(const GArgs *g, int n, double beta);
  // C = beta C + sum_s A_s B_s^T over up to 4 segments with the same M, N and
  // output (each its own K): one multi-segment tensor-core launch when every
  // segment takes the split path, else one G call per segment
  struct Seg {
    const double *A;
    long long lda;
    const double *B;
    long long ldb;
    int K;
    bool constA, constB;
  };
  int Gmulti(int M, int N, const Seg *sg, int nseg, double beta, const CView &C);

  // Lambda (adjoint) state: lambda = [l1 | l2] like X, dE/dT, tape
  DBuf L, Ln, gE, lrhs;
  bool have_amplitudes = false, have_lambda = false;
  std::vector<TapeOp> tape;
  bool recording = false;
  std::vector<DBuf *> active;
  std::map<DBuf *, DBuf> adjoint;
  // transposes of constant operands, by (source, rows, cols, leading
  // dimension): one array can be the operand of contractions of several shapes
  std::map<std::tuple<const double *, int, int, long long>, DBuf> tcache;
  // transposes of the recorded forward values the backward pass reads: fixed
  // while the tape is (every Lambda iteration and EOM product replays the
  // same tape), dropped with their cached splits when a pass is recorded
  std::map<std::tuple<const double *, int, int, long long>, DBuf> tape_tcache;
  const double *tape_transposed(const double *src, int rows, int cols, long long ld);
  void tape_cache_clear();
  std::vector<const double *> symmetric;     // constant matrices equal to their transpose
  DBuf bwdA, bwdB, bwdC, bwdD;
  std::vector<DBuf *> registry();
  DBuf *owner(const void *p);
  bool is_active(const void *p);
  void mark_active(const void *p);
  double *adj(const void *p);
  int tmp(DBuf &b, size_t n);
  const double *transposed(const double *src, int rows, int cols, long long ld, bool cst,
                           DBuf &scratch);
  int backward();
  void zero_adjoints();
  int record_residual(bool fock_active);
  int tau_op(double *out, const double *t2, const double *t1, double c);
  int lambda_rhs();
  // EOM-EE: sigma = P (dZ/dT)^T x - D o x on the excitations of irrep h
  // (needs record_residual at the converged amplitudes first)
  int eom_sigma(const double *x, double *out, int h, const int *d_irr_o, const int *d_irr_v);
  int density(std::vector<double> &D);

  // statistics
  long long gemm_calls = 0;
  double gemm_flops = 0.0;
  cudaEvent_t ev_lad0 = nullptr, ev_lad1 = nullptr;  // around the pp-ladder contraction

  ~CCEngine();
  int alloc(DBuf &b, size_t n);
  int load_from_lists();
  int setup_intermediates();
  int mp2_guess();
  // TGUESS restart (vcc/drdtgss.F): T1 from list 90, T2 from list 46 when both
  // exist with this system's dimensions; *read = false leaves X untouched
  int read_guess(bool *read);
  int residual();   // Z1, Z2 from X
  int iteration(int icycle, int exporder, double *e_out3, double *res, double *dres,
                bool *extrap, bool lambda = false);
  int write_back();
  int write_amplitudes(const double *a1, const double *a2, int list1, int list2ab, int list2aa);
  // (T), trp/trps2.F: the triplets t with t % nranks == rank (partial sums)
  int triples(double *e4, double *e5, double *seconds, int rank = 0, int nranks = 1);
  void release();

  // contraction dispatch (FP64 DMMA or BF16x3 tcgen05)
  int G(int M, int N, int K, double alpha, const double *A, long long lda, const double *B,
        long long ldb, double beta, const CView &C, bool constA = false, bool constB = false);
  int perm(double *out, int n0, int n1, int n2, int n3, double beta,
           std::initializer_list<PermTerm> terms);
  int copy(double *dst, const double *src, size_t n);
};

constexpr long long kHugeView = 1LL << 62;  // CView divisor meaning "no split"

// Device tables mapping the dense [p,q,r,s] index space of one DPD list onto
// its irrep blocks (pair indices, signs, orbital irreps, block pointers).
struct DevMap {
  int *d_rowidx = nullptr, *d_colidx = nullptr;
  signed char *d_rowsgn = nullptr, *d_colsgn = nullptr;
  int *d_irr[4] = {nullptr, nullptr, nullptr, nullptr};
  double **d_base = nullptr;
  int *d_nrows = nullptr;
  DpdMap m;
  DevMap() = default;
  DevMap(const DevMap &) = delete;
  DevMap &operator=(const DevMap &) = delete;
  ~DevMap();
};
// Tables of list `list` (row pair type typeL, column pair type typeR; with
// create the list is first touched through INIPCK) for occupied / virtual
// orbitals of the given irreps, in DPD order.
int make_map(DevMap &dm, int list, int typeL, int typeR, const std::vector<int> &irr_o,
             const std::vector<int> &irr_v, bool create);

int accept_update(CCEngine &E, bool extrap, int ndimr, bool lambda);
CCEngine *engine_instance(bool create);
void engine_reset();

}  // namespace acesb200
