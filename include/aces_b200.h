/*
 * aces_b200.h -- C-ABI of the B200 coupled-cluster engine (CCSD / (T) / Lambda).
 *
 * The entry points mirror the reference's list/record interface and member
 * programs so that a Fortran or C host can bind them one-for-one.  Every
 * function returns an int status (ACES_OK = 0, negative on error) where the
 * reference calls aces_exit(); no function terminates the process.
 *
 * Conventions shared with the reference:
 *   - irreps, list ids and column indices are 1-based (Fortran style);
 *   - a list is a set of 2-D column-major arrays, one per irrep; column c of
 *     irrep h holds nrows(h) doubles (acescore/aces_list_touch.F);
 *   - pair types 1..25 and their packing (PACK a<b, PCK2 a<=b, FULL) follow
 *     acescore/aces_com_symloc.F; IRPDPD(irrep,type) follows
 *     acescore/aces_com_sympop.F; DIRPRD is the XOR product of 0-based irreps.
 *   - all list data live in device memory (one arena per process); the plain
 *     GETLST/PUTLST entry points stage through host memory like the
 *     reference's file I/O, the *_dev variants copy device-to-device.
 */
#ifndef ACES_B200_H
#define ACES_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

enum {
  ACES_OK = 0,
  ACES_ERR_ARG = -1,        /* invalid argument (bad irrep, list, bounds)      */
  ACES_ERR_NOLIST = -2,     /* list/irrep not touched                          */
  ACES_ERR_REDIM = -3,      /* re-touch with different dims (aces_list_touch.F:83) */
  ACES_ERR_CUDA = -4,       /* CUDA runtime error                              */
  ACES_ERR_NOMEM = -5,      /* device allocation failed (INSMEM)               */
  ACES_ERR_NOREC = -6,      /* JOBARC record absent (getrec.F)                 */
  ACES_ERR_NOSYM = -7,      /* symmetry not initialised                        */
  ACES_ERR_SINGULAR = -8,   /* DIIS bordered system singular (libr/dodiis.F:49) */
  ACES_ERR_NOCONV = -9,     /* CC equations did not converge (vcc/vcc.F:1439)  */
  ACES_ERR_NAN = -10,       /* non-finite amplitudes or energy                 */
  ACES_ERR_TIMEOUT = -11,   /* a bounded device wait gave up                   */
  ACES_ERR_UNSUPPORTED = -12
};

/* ---- runtime ---------------------------------------------------------- */

/* aces_init (acescore/aces_init.F): select the CUDA device, reset lists and
 * records.  Safe to call again (re-initialises). */
int aces_init(int device);
/* aces_fin (acescore/aces_fin.F): free every list and record. */
int aces_fin(void);
/* Last error message (static storage). */
const char *aces_last_error(void);
/* Device-memory accounting of the library's caching allocator (no
 * counterpart in the reference, whose ICORE heap is one up-front malloc,
 * acescore/aces_malloc.c:48): alloc_calls counts every device buffer the
 * library has requested since load, driver_allocs the requests the cache
 * could not serve (cudaMalloc calls), cached_bytes the released memory held
 * for reuse.  Any pointer may be NULL. */
int aces_pool_stats(long long *alloc_calls, long long *driver_allocs, long long *cached_bytes);

/* ---- symmetry / DPD metadata ------------------------------------------- */

/* Replaces the JOBARC-driven set-up of /SYMINF/, /SYM/, /SYMPOP/ and
 * /SYMLOC/ (acescore/aces_com_syminf.F, aces_com_sym.F, aces_com_sympop.F,
 * aces_com_symloc.F) for a closed-shell (RHF) reference: pop[h] occupied and
 * vrt[h] virtual orbitals per irrep, h = 0..nirrep-1, alpha = beta. */
int aces_sym_init(int nirrep, const int *pop, const int *vrt);
/* IRPDPD(irrep, type): number of pairs of pair type `type` (1..22) whose
 * product irrep is `irrep` (include/sympop.com). */
int aces_irpdpd(int irrep, int type);
/* ISYMOFF(irrep_q, irrep_pq, type): 1-based offset of the (irrep_p, irrep_q)
 * block inside the pairs of total irrep irrep_pq (include/symloc.com). */
int aces_isymoff(int irrep_q, int irrep_pq, int type);
/* DIRPRD(i, j) (include/syminf.com). */
int aces_dirprd(int i, int j);

/* ---- lists (MOINTS / GAMLAM files) -------------------------------------- */

/* ACES_LIST_TOUCH (acescore/aces_list_touch.F:24): create list `list`, irrep
 * `irrep` with nrows x ncols doubles, zero-filled.  Re-touching with the same
 * dims is a no-op; different dims return ACES_ERR_REDIM. */
int aces_list_touch(int ncols, int nrows, int irrep, int list, int nofrag);
/* UPDMOI (libr/updmoi.F:11): same as aces_list_touch. */
int aces_updmoi(int ncols, int nrows, int irrep, int list, int iarg1, int iarg2);
/* INIPCK (libr/inipck.F:4): touch every irrep of `list` with rows of pair type
 * sytypl (irrep DIRPRD(irrepr, irrepx)) and columns of pair type sytypr
 * (irrep irrepr); with iset != 0 record ISYTYP(1:2, list). */
int aces_inipck(int irrepx, int sytypl, int sytypr, int list, int iset);
/* ISYTYP(1|2, list). */
int aces_isytyp(int which, int list);
/* Dimensions of one list irrep (0 rows/cols when untouched). */
int aces_list_dims(int irrep, int list, int *ncols, int *nrows);
/* GETLST (acescore/getlst.F:19): copy columns first..first+ncols-1 of
 * (irrep, list) into host memory `dst` (column-major). */
int aces_getlst(double *dst, int first, int ncols, int irrep, int list);
/* PUTLST (acescore/putlst.F:19): the mirror of GETLST. */
int aces_putlst(const double *src, int first, int ncols, int irrep, int list);
/* Device-pointer variants (stream 0 ordered, asynchronous w.r.t. the host). */
int aces_getlst_dev(double *dst, int first, int ncols, int irrep, int list);
int aces_putlst_dev(const double *src, int first, int ncols, int irrep, int list);
/* GETALL / PUTALL (acesutil/getall.F, acesutil/putall.f): all irreps
 * r = 1..nirrep of a list whose column irrep is r, concatenated; `len` is the
 * expected total length in doubles (checked). */
int aces_getall(double *dst, long long len, int irrepx, int list);
int aces_putall(const double *src, long long len, int irrepx, int list);
/* ACES_LIST_MEMSET (acescore/aces_list_memset.F): byte fill of one irrep. */
int aces_list_memset(int irrep, int list, int byte);
/* Device address of (irrep, list) column 1, or NULL. */
double *aces_list_devptr(int irrep, int list);

/* The integral lists the CC programs read, produced on the device (the
 * reference's vtran + intprc chain, intprc/clmoio.F:46-260, for
 * density-fitted or Cholesky-decomposed MO integrals): from the factors
 * B[L][p][q] (naux x nmo x nmo doubles, C order, symmetric in p and q,
 * orbitals in DPD order -- occupied by irrep, then virtual by irrep -- with
 * (pq|rs) = sum_L B[L][p][q] B[L][r][s]) it creates lists 13 <Ij|Kl>,
 * 10 <Ij|Ka>, 16 <Ab|Ij>, 25 <Ai|Bj>, 30 <Ab|Ci> and 233 <Ab|Cd> in every irrep
 * (INIPCK) and fills them in FP64.  `B` is a device pointer when on_device is
 * nonzero, else host memory copied in.  Requires aces_sym_init; the orbital
 * energies (record SCFEVALA) are the caller's, as with PUTLST. */
int aces_intprc_df(const double *B, int naux, int on_device);

/* ---- records (JOBARC) --------------------------------------------------- */

/* PUTREC / GETREC (acescore/putrec.F, acescore/getrec.F): named byte
 * vectors.  getrec fails with ACES_ERR_NOREC when absent and ACES_ERR_ARG when
 * nbytes exceeds the stored length. */
int aces_putrec(const char *label, long long nbytes, const void *buf);
int aces_getrec(const char *label, long long nbytes, void *buf);
long long aces_reclen(const char *label);

/* ---- BLAS boundary ------------------------------------------------------ */

/* XGEMM (tools/xgemm.F:10-49, crust/xgemm.F:10-51): column-major
 * C = alpha * op(A) op(B) + beta * C on DEVICE pointers, op = 'N' or 'T'
 * (case-insensitive); quick return when m*n == 0.  `precision` selects the
 * FP64 DMMA kernel or the BF16x3 tcgen05 kernel (ACES_PREC_*).  Synchronous. */
int aces_xgemm(char transa, char transb, int m, int n, int k, double alpha, const double *A,
               int lda, const double *B, int ldb, double beta, double *Cmat, int ldc,
               int precision);

/* The same FP64 product for callers that cannot allocate device memory (no
 * counterpart in the reference): hosts that gave all device memory to their
 * own allocator at start-up, or callers that must not pay an allocation's
 * implicit synchronisation.  It calls no cudaMalloc/cudaFree and no
 * allocating library routine: its scratch (m*k doubles when transa = 'N',
 * n*k when transb = 'T', plus optional split-K partials) comes from one
 * static device array of 2^20 doubles (8 MiB) that every GPU loading the
 * library holds until exit; larger requests return ACES_ERR_ARG.  The first
 * call on each device looks up the array's device address (set-up); make
 * that first call before any stream capture.  Every call runs on the legacy
 * default stream of the current device and returns when the product is
 * done.  Calls share the array: calls that overlap on the GPU race.  FP64
 * only. */
int aces_xgemm_static(char transa, char transb, int m, int n, int k, double alpha,
                      const double *A, int lda, const double *B, int ldb, double beta,
                      double *Cmat, int ldc);

/* Bound on every device-side wait of the tensor-core contraction kernels on
 * the current device (default 4 s; (0, 60] accepted).  A kernel whose wait
 * runs out records it, waits (again bounded) for the copies and products it
 * issued, releases its tensor memory and returns; the calling entry point
 * then returns ACES_ERR_TIMEOUT.  No counterpart in the reference (its BLAS
 * calls cannot stall on a device). */
int aces_set_wait_limit(double seconds);
/* Test hook for that path (no counterpart in the reference): mode 1 makes the
 * copy-issuing thread of the tensor-core kernels on the current device issue
 * nothing, so every product waits out the limit above and the call reports
 * ACES_ERR_TIMEOUT with no copy or product in flight; mode 0 restores normal
 * operation. */
int aces_debug_inject(int mode);
/* Tile variant of the tensor-core contractions (no counterpart in the
 * reference): 1 = products of at least 256 rows run on CTA pairs (tcgen05
 * cta_group::2, 256 x 128 tiles), 0 = one CTA per 128 x 144 tile (the
 * default, faster on B200 for the CC contractions).  Both give the same
 * error bound; process-wide. */
int aces_set_tc_pairs(int on);
/* Tile width of the tensor-core launches whose every output tile is one
 * accumulation chunk with FP32 output and 144 < N <= 256 (the batched (T)
 * classes for 144 < v <= 192; no counterpart in the reference): 1 = one
 * 128 x 256 tile across N (the default), 0 = 128 x 144 tiles.  Same
 * arithmetic either way; process-wide. */
int aces_set_tc_wide(int on);
/* Tile autotuner of the tensor-core contractions (no counterpart in the
 * reference; the reference's XGEMM calls take whatever its BLAS does).
 * mode 1: the first product of each shape class on a device times the tile
 * variants that apply to it -- one CTA per tile or CTA pairs and split K or
 * not for single and grouped products, 144- or 256-wide tiles for the
 * FP32-output batched (T) launches -- with CUDA
 * events on the product's stream (the call then waits for the device), and
 * later products of the class reuse the fastest; mode 0 (default): the
 * built-in rules; mode 2: forget every cached choice (the on/off state is
 * kept).  A class is the launch kind, segment count, output type and the
 * tile and k-tile counts to two significant bits.  No tuning while the
 * stream is being captured; trial runs write the product's own output when
 * beta = 0, else a scratch array from the library's allocator.  Every
 * variant meets the same error bound.  Process-wide. */
int aces_set_autotune(int mode);
/* Shape classes tuned so far, how many of them chose a variant other than
 * the built-in rule, and the device ms the timed trial runs took. */
int aces_autotune_stats(long long *classes, long long *changed, double *tune_ms);
/* The current device's cached tile choices to a text file, and back (no
 * counterpart in the reference).  Loading replaces the classes the file
 * names (for the current device; later products of those classes launch
 * the loaded choice without timing, whether or not tuning is on) and
 * rejects a file with any line that is not a choice the tuner could make
 * (ACES_ERR_ARG, nothing loaded).  A host that loads one saved tuning in
 * every run gets the same tile variant per class in every run. */
int aces_autotune_save(const char *path);
int aces_autotune_load(const char *path);

/* ---- member programs ---------------------------------------------------- */

/* Precision of the tensor contractions. */
enum {
  ACES_PREC_FP64 = 0,      /* FP64 everywhere (the plain GPU path)            */
  ACES_PREC_BF16X3 = 1     /* split BF16x3 tcgen05 products, FP32 accumulate,
                              FP64 denominators / DIIS / energies / norms     */
};

/* Job parameters: the IFLAGS fields the CC programs read (include/flags.h).
 * Inputs are the lists and records named at each entry point below;
 * outputs are written back to lists 46/44 (T2), 90 (T1) and records. */
typedef struct aces_cc_config {
  int cc_conv;        /* IFLAGS(4): converge when max |dT| < 10^-cc_conv     */
  int cc_maxcyc;      /* IFLAGS(7)                                           */
  int cc_exporder;    /* IFLAGS(12): DIIS subspace (<= 25)                   */
  int precision;      /* ACES_PREC_*                                         */
  int triples;        /* 1: run (T) after CCSD (CALC=CCSD(T))                */
  int use_graph;      /* 1: the residual pass of every cycle after the second
                         is a replay of a CUDA graph captured on the second
                         (the ladder stays timed through external event
                         nodes of the graph)                                 */
  int verbose;        /* 1: per-iteration log on stdout (IFLAGS(1))          */
  int timing_warmup;  /* cycles excluded from the timing outputs             */
  /* outputs */
  double e_ccsd;      /* correlation energy of the final amplitudes          */
  double e_t4;        /* E[4]T                                               */
  double e_st5;       /* E[5]ST                                              */
  double last_residual;
  int ncycle;
  int converged;
  double seconds_per_iter;   /* mean device time of a timed cycle (CUDA events) */
  double seconds_triples;    /* device time of (T)                           */
  double seconds_ladder;     /* mean device time of the particle-particle ladder
                                contraction in a timed cycle                 */
  double flops_per_iter;     /* flops of all contractions of one cycle       */
  long long launches_per_iter; /* kernels launched in one timed cycle        */
  double seconds_setup;      /* device time reading lists and resorting integrals */
  /* (T) over several GPUs (inputs): this call evaluates the occupied triplets
   * i >= j >= k whose index t in the order (i, then j <= i, then k <= j)
   * satisfies t % triples_nranks == triples_rank, and e_t4 / e_st5 are that
   * shard's partial sums (add them over the ranks).  0 / 0 or 0 / 1: all. */
  int triples_rank;
  int triples_nranks;
  /* DAMP_CC (vcc/vcc.F:71, IFLAGS2 damp_cc x 0.01; vcc/damp_cc_residual.F):
   * after the denominator division the new amplitudes become
   * T_old + damp (T_new - T_old); convergence is judged on the undamped
   * difference (vcc/dodiis0.F:93-97).  0 or 1: no damping. */
  double damp;
  /* TGUESS restart (vcc/drdtgss.F): on input 1 starts from the amplitudes in
   * lists 90 (T1) and 46 (T2, AB) -- a previous xvcc_run's output or the
   * caller's -- instead of the MP2 guess, when both lists exist with this
   * system's dimensions; on output 1 if they were read, 0 if the MP2 guess
   * was used. */
  int tguess;
} aces_cc_config;

/* PROGRAM VCC (vcc/vcc.F:9): RHF CCSD (and (T) when cfg->triples).  Reads
 * lists 13, 10, 16, 25, 30, 233 and records SCFEVALA (orbital energies, DPD
 * order) plus, for a non-Hartree-Fock Fock matrix, record FOCKMAT; writes T1
 * to list 90 (irrep 1), T2(AB) to list 46, T2(AA) to list 44 and record
 * TOTENERG-style records CCSDENRG, E4T, E5ST. */
int xvcc_run(aces_cc_config *cfg);

/* PROGRAM VLAMCC (lambda/vlamcc.F): Lambda equations for the amplitudes left
 * by xvcc_run; writes L1 to list 190 (irrep 1), L2(AB) to list 146 and
 * L2(AA) = L2 - L2~ to list 144, in the reference's convention (the
 * multipliers its own xlambda leaves there: L1 = l1/2, L2 = (2 l2 + l2~)/3 of
 * the Lagrange multipliers l of the spin-adapted residual). */
int xlambda_run(aces_cc_config *cfg);

/* DENSOO/DENSVV/DENSVO (dens/densoo.F, densvv.F, densvo.F): the CCSD
 * one-particle density from T and Lambda, written to record DENSMAT (nmo x
 * nmo, DPD orbital order, row-major). */
int xdens_1pdm(aces_cc_config *cfg);

/* Excited states (PROGRAM VEE, vee/doeomee_david.F): singlet EOM-EE-CCSD
 * excitation energies of a closed-shell reference, nroots[h] lowest roots of
 * every irrep h + 1 (ESTATE_SYM), found by a Davidson iteration from the
 * single excitations of smallest orbital-energy gap. */
typedef struct aces_eom_config {
  int nroots[8];       /* roots per irrep, 0..8                               */
  int eom_conv;        /* converged when |residual| and |d omega| < 10^-eom_conv */
  int eom_maxcyc;      /* Davidson iterations per irrep                       */
  int max_subspace;    /* trial vectors kept before a collapse (0: 40)        */
  int precision;       /* ACES_PREC_*                                         */
  int verbose;
  /* outputs */
  double omega[8][8];  /* excitation energies (Eh), [irrep][root], ascending  */
  int converged[8];
  int niter[8];
  int nsigma;          /* products with the Jacobian evaluated                */
  double seconds;
} aces_eom_config;

/* EOM-EE-CCSD on the amplitudes left by xvcc_run: the singlet excitation
 * energies are the eigenvalues of the CC Jacobian on the pair-symmetric
 * amplitude space, found from its transpose (the reverse replay of the
 * residual pass that the Lambda equations use).  Writes record EOMEXCIT
 * (64 doubles, [irrep][root]). */
int xvee_run(aces_eom_config *cfg);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* ACES_B200_H */
