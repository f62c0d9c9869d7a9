"""Python binding of the B200 coupled-cluster engine (C-ABI in include/aces_b200.h).

The engine is the shared library ``libacesb200.so`` built next to this file
(``python aces-ii_b200/build.py``).  Loading fails loudly when it is absent:
there is no CPU fallback.

Typical use mirrors the reference's program flow (intprc writes the MO
integral lists, xvcc reads them, vcc/vcc.F):

    import acesb200 as ab
    lib = ab.load()
    lib.init(0)
    lib.sym_init(pop, vrt)
    ab.put_hamiltonian(lib, eps, blocks, irr_o, irr_v)   # lists 13, 10, 16, 25, 30, 233
    res = lib.xvcc(cc_conv=7, cc_exporder=5)
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .dpd import DPD, put_dense_list, get_dense_list  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "libacesb200.so")

ACES_OK = 0
PREC_FP64 = 0
PREC_BF16X3 = 1

# exported C-ABI symbols (include/aces_b200.h)
SYMBOLS = [
    "aces_init", "aces_fin", "aces_last_error", "aces_pool_stats", "aces_sym_init", "aces_irpdpd",
    "aces_isymoff", "aces_dirprd", "aces_list_touch", "aces_updmoi", "aces_inipck",
    "aces_isytyp", "aces_list_dims", "aces_getlst", "aces_putlst", "aces_getlst_dev",
    "aces_putlst_dev", "aces_getall", "aces_putall", "aces_list_memset", "aces_list_devptr",
    "aces_intprc_df",
    "aces_putrec", "aces_getrec", "aces_reclen", "aces_xgemm", "aces_xgemm_static",
    "aces_set_wait_limit", "aces_debug_inject", "aces_set_tc_pairs", "aces_set_tc_wide", "aces_set_autotune", "aces_autotune_stats", "aces_autotune_save", "aces_autotune_load", "xvcc_run", "xlambda_run", "xdens_1pdm",
    "xvee_run",
]


class CCConfig(C.Structure):
    """aces_cc_config (include/aces_b200.h)."""
    _fields_ = [
        ("cc_conv", C.c_int), ("cc_maxcyc", C.c_int), ("cc_exporder", C.c_int),
        ("precision", C.c_int), ("triples", C.c_int), ("use_graph", C.c_int),
        ("verbose", C.c_int), ("timing_warmup", C.c_int),
        ("e_ccsd", C.c_double), ("e_t4", C.c_double), ("e_st5", C.c_double),
        ("last_residual", C.c_double), ("ncycle", C.c_int), ("converged", C.c_int),
        ("seconds_per_iter", C.c_double), ("seconds_triples", C.c_double),
        ("seconds_ladder", C.c_double), ("flops_per_iter", C.c_double),
        ("launches_per_iter", C.c_longlong), ("seconds_setup", C.c_double),
        ("triples_rank", C.c_int), ("triples_nranks", C.c_int),
        ("damp", C.c_double), ("tguess", C.c_int),
    ]


class EOMConfig(C.Structure):
    """aces_eom_config (include/aces_b200.h)."""
    _fields_ = [
        ("nroots", C.c_int * 8), ("eom_conv", C.c_int), ("eom_maxcyc", C.c_int),
        ("max_subspace", C.c_int), ("precision", C.c_int), ("verbose", C.c_int),
        ("omega", (C.c_double * 8) * 8), ("converged", C.c_int * 8), ("niter", C.c_int * 8),
        ("nsigma", C.c_int), ("seconds", C.c_double),
    ]


class AcesError(RuntimeError):
    def __init__(self, fn, status, msg):
        super().__init__(f"{fn} returned {status}: {msg}")
        self.status = status


_DP = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class Lib:
    """Thin checked wrapper over the shared library."""

    def __init__(self, path=LIBPATH):
        if not os.path.exists(path):
            raise FileNotFoundError(
                f"{path} is missing: build it with `python aces-ii_b200/build.py` "
                "(the engine has no CPU fallback)")
        self.path = path
        self.h = C.CDLL(path)
        h = self.h
        h.aces_last_error.restype = C.c_char_p
        h.aces_list_devptr.restype = C.c_void_p
        h.aces_list_devptr.argtypes = [C.c_int, C.c_int]
        h.aces_reclen.restype = C.c_longlong
        h.aces_reclen.argtypes = [C.c_char_p]
        h.aces_getlst.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]
        h.aces_putlst.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]
        h.aces_getall.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.c_int]
        h.aces_putall.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.c_int]
        h.aces_putrec.argtypes = [C.c_char_p, C.c_longlong, C.c_void_p]
        h.aces_getrec.argtypes = [C.c_char_p, C.c_longlong, C.c_void_p]
        h.aces_sym_init.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        h.aces_xgemm.argtypes = [C.c_char, C.c_char, C.c_int, C.c_int, C.c_int, C.c_double,
                                 C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_double,
                                 C.c_void_p, C.c_int, C.c_int]
        h.aces_xgemm_static.argtypes = [C.c_char, C.c_char, C.c_int, C.c_int, C.c_int,
                                        C.c_double, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                        C.c_double, C.c_void_p, C.c_int]
        for fn in ("xvcc_run", "xlambda_run", "xdens_1pdm"):
            getattr(h, fn).argtypes = [C.POINTER(CCConfig)]
        h.xvee_run.argtypes = [C.POINTER(EOMConfig)]

    def _chk(self, fn, status):
        if status != ACES_OK:
            raise AcesError(fn, status, self.h.aces_last_error().decode())
        return status

    def error(self):
        return self.h.aces_last_error().decode()

    def pool_stats(self):
        """(device buffers requested, cudaMalloc calls, cached bytes) of the
        library's caching allocator since load."""
        a, d, c = C.c_longlong(), C.c_longlong(), C.c_longlong()
        self._chk("aces_pool_stats",
                  self.h.aces_pool_stats(C.byref(a), C.byref(d), C.byref(c)))
        return a.value, d.value, c.value

    # ---- runtime / symmetry -------------------------------------------------
    def init(self, device=0):
        self._chk("aces_init", self.h.aces_init(device))

    def fin(self):
        self._chk("aces_fin", self.h.aces_fin())

    def sym_init(self, pop, vrt):
        n = len(pop)
        p = (C.c_int * n)(*[int(x) for x in pop])
        v = (C.c_int * n)(*[int(x) for x in vrt])
        self._chk("aces_sym_init", self.h.aces_sym_init(n, p, v))
        self.nirrep = n
        self.pop = [int(x) for x in pop]
        self.vrt = [int(x) for x in vrt]

    def irpdpd(self, irrep, typ):
        r = self.h.aces_irpdpd(irrep, typ)
        if r < 0:
            raise AcesError("aces_irpdpd", r, self.error())
        return r

    def isymoff(self, irrep_q, irrep_pq, typ):
        r = self.h.aces_isymoff(irrep_q, irrep_pq, typ)
        if r < 0:
            raise AcesError("aces_isymoff", r, self.error())
        return r

    # ---- lists ------------------------------------------------------------------
    def inipck(self, irrepx, typl, typr, lst, iset=1):
        self._chk("aces_inipck", self.h.aces_inipck(irrepx, typl, typr, lst, iset))

    def list_touch(self, ncols, nrows, irrep, lst):
        return self.h.aces_list_touch(ncols, nrows, irrep, lst, 0)

    def list_dims(self, irrep, lst):
        nc, nr = C.c_int(), C.c_int()
        self._chk("aces_list_dims", self.h.aces_list_dims(irrep, lst, C.byref(nc), C.byref(nr)))
        return nr.value, nc.value

    def getlst(self, first, ncols, irrep, lst):
        nr, _ = self.list_dims(irrep, lst)
        out = np.zeros((ncols, nr))  # column-major: each row of `out` is one column
        self._chk("aces_getlst", self.h.aces_getlst(out.ctypes.data, first, ncols, irrep, lst))
        return out.T

    def putlst(self, cols, first, irrep, lst):
        """cols: (nrows, ncols) array; stored column-major."""
        a = np.ascontiguousarray(np.asarray(cols, dtype=np.float64).T)
        ncols = a.shape[0]
        self._chk("aces_putlst", self.h.aces_putlst(a.ctypes.data, first, ncols, irrep, lst))

    def putlst_raw(self, buf, first, ncols, irrep, lst):
        """buf: contiguous float64 buffer already in column-major order."""
        self._chk("aces_putlst", self.h.aces_putlst(buf.ctypes.data, first, ncols, irrep, lst))

    def getall(self, length, irrepx, lst):
        out = np.zeros(length)
        self._chk("aces_getall", self.h.aces_getall(out.ctypes.data, length, irrepx, lst))
        return out

    def putall(self, vec, irrepx, lst):
        a = np.ascontiguousarray(vec, dtype=np.float64)
        self._chk("aces_putall", self.h.aces_putall(a.ctypes.data, a.size, irrepx, lst))

    def intprc_df(self, B, naux=None, on_device=None):
        """Lists 13, 10, 16, 25, 30, 233 from MO factors B[L, p, q] (DPD orbital
        order) built on the device (aces_intprc_df).  ``B`` is a numpy array
        (host), a torch tensor (host or CUDA) or a raw device pointer with
        ``naux`` given."""
        if isinstance(B, int):
            if naux is None:
                raise ValueError("naux is required with a raw pointer")
            ptr, dev = B, 1 if on_device is None else int(on_device)
        elif isinstance(B, np.ndarray):
            B = np.ascontiguousarray(B, dtype=np.float64)
            self._keep = B
            ptr, dev, naux = B.ctypes.data, 0, B.shape[0]
        else:   # torch tensor
            if not B.is_contiguous() or str(B.dtype) != "torch.float64":
                raise ValueError("B must be a contiguous float64 tensor")
            ptr, dev, naux = B.data_ptr(), int(B.is_cuda), B.shape[0]
        self._chk("aces_intprc_df", self.h.aces_intprc_df(C.c_void_p(ptr), int(naux), dev))

    # ---- records ------------------------------------------------------------------
    def putrec(self, label, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        self._chk("aces_putrec", self.h.aces_putrec(label.encode(), a.nbytes, a.ctypes.data))

    def getrec(self, label, n):
        out = np.zeros(n)
        self._chk("aces_getrec", self.h.aces_getrec(label.encode(), out.nbytes, out.ctypes.data))
        return out

    # ---- BLAS boundary ---------------------------------------------------------------
    def xgemm(self, transa, transb, m, n, k, alpha, A_ptr, lda, B_ptr, ldb, beta, C_ptr, ldc,
              precision=PREC_FP64):
        """XGEMM on device pointers (column-major, tools/xgemm.F)."""
        self._chk("aces_xgemm", self.h.aces_xgemm(transa.encode(), transb.encode(), m, n, k,
                                                  alpha, A_ptr, lda, B_ptr, ldb, beta, C_ptr,
                                                  ldc, precision))

    def xgemm_static(self, transa, transb, m, n, k, alpha, A_ptr, lda, B_ptr, ldb, beta, C_ptr,
                     ldc):
        """FP64 XGEMM that allocates no device memory (static scratch); see
        aces_xgemm_static in include/aces_b200.h."""
        self._chk("aces_xgemm_static",
                  self.h.aces_xgemm_static(transa.encode(), transb.encode(), m, n, k, alpha,
                                           A_ptr, lda, B_ptr, ldb, beta, C_ptr, ldc))

    def set_wait_limit(self, seconds):
        """Bound of the tensor-core kernels' device-side waits (aces_set_wait_limit)."""
        self._chk("aces_set_wait_limit", self.h.aces_set_wait_limit(C.c_double(seconds)))

    def set_tc_pairs(self, on):
        """Tensor-core tile variant: 1 = CTA pairs for products of >= 256 rows
        (aces_set_tc_pairs), 0 = one CTA per tile (default)."""
        self._chk("aces_set_tc_pairs", self.h.aces_set_tc_pairs(int(on)))

    def set_tc_wide(self, on):
        """Tile width of the single-chunk FP32-output launches: 1 = 128 x 256
        (aces_set_tc_wide, default), 0 = 128 x 144."""
        self._chk("aces_set_tc_wide", self.h.aces_set_tc_wide(int(on)))

    def set_autotune(self, mode):
        """Tile autotuner (aces_set_autotune): 1 = time the applicable tile
        variants on the first product of each shape class and reuse the
        fastest, 0 = built-in rules (default), 2 = forget the cached choices."""
        self._chk("aces_set_autotune", self.h.aces_set_autotune(int(mode)))

    def autotune_stats(self):
        """(classes tuned, classes that left the built-in rule, device ms of
        the timed trial runs) -- aces_autotune_stats."""
        n, c, ms = C.c_longlong(), C.c_longlong(), C.c_double()
        self._chk("aces_autotune_stats",
                  self.h.aces_autotune_stats(C.byref(n), C.byref(c), C.byref(ms)))
        return n.value, c.value, ms.value

    def autotune_save(self, path):
        """The current device's cached tile choices to a text file (aces_autotune_save)."""
        self._chk("aces_autotune_save", self.h.aces_autotune_save(str(path).encode()))

    def autotune_load(self, path):
        """Tile choices from a file saved by autotune_save (aces_autotune_load)."""
        self._chk("aces_autotune_load", self.h.aces_autotune_load(str(path).encode()))

    def debug_inject(self, mode):
        """Test hook: 1 = the tensor-core producer issues no copies (aces_debug_inject)."""
        self._chk("aces_debug_inject", self.h.aces_debug_inject(mode))

    # ---- programs -----------------------------------------------------------------
    def _run(self, fn, cfg, allow_noconv=False):
        st = getattr(self.h, fn)(C.byref(cfg))
        if st != ACES_OK and not (allow_noconv and st == -9):
            raise AcesError(fn, st, self.error())
        return cfg

    def xvcc(self, cc_conv=7, cc_maxcyc=50, cc_exporder=5, precision=PREC_FP64, triples=0,
             use_graph=0, verbose=0, allow_noconv=False, timing_warmup=0, triples_rank=0,
             triples_nranks=1, damp=1.0, tguess=0):
        cfg = CCConfig(cc_conv=cc_conv, cc_maxcyc=cc_maxcyc, cc_exporder=cc_exporder,
                       precision=precision, triples=triples, use_graph=use_graph,
                       verbose=verbose, timing_warmup=timing_warmup, triples_rank=triples_rank,
                       triples_nranks=triples_nranks, damp=damp, tguess=tguess)
        return self._run("xvcc_run", cfg, allow_noconv)

    def xlambda(self, cc_conv=7, cc_maxcyc=50, cc_exporder=5, precision=PREC_FP64, verbose=0,
                timing_warmup=0):
        cfg = CCConfig(cc_conv=cc_conv, cc_maxcyc=cc_maxcyc, cc_exporder=cc_exporder,
                       precision=precision, verbose=verbose, timing_warmup=timing_warmup)
        return self._run("xlambda_run", cfg)

    def xdens(self):
        return self._run("xdens_1pdm", CCConfig())

    def xvee(self, nroots, eom_conv=7, eom_maxcyc=60, max_subspace=0, precision=PREC_FP64,
             verbose=0):
        """Singlet EOM-EE-CCSD excitation energies (Eh) of the lowest nroots[h]
        states of every irrep h (xvee_run); returns (config, {irrep: [omega]})."""
        n = [int(x) for x in nroots] + [0] * (8 - len(nroots))
        cfg = EOMConfig(eom_conv=eom_conv, eom_maxcyc=eom_maxcyc, max_subspace=max_subspace,
                        precision=precision, verbose=verbose)
        for h in range(8):
            cfg.nroots[h] = n[h]
        st = self.h.xvee_run(C.byref(cfg))
        if st != ACES_OK:
            raise AcesError("xvee_run", st, self.error())
        return cfg, {h: [cfg.omega[h][r] for r in range(n[h])] for h in range(8) if n[h]}


_lib = None


def load(path=LIBPATH):
    global _lib
    if _lib is None or _lib.path != path:
        _lib = Lib(path)
    return _lib


# Integral lists read by xvcc_run: list id -> (row pair type, column pair type,
# physicists' block and the transpose taking it to [row p, row q, col r, col s]).
INTEGRAL_LISTS = {
    13: (14, 14, "oooo", (0, 1, 2, 3)),    # <Ij|Kl>
    10: (14, 18, "ooov", (0, 1, 2, 3)),    # <Ij|Ka>
    16: (13, 14, "oovv", (2, 3, 0, 1)),    # <Ab|Ij>
    25: (11, 11, "ovov", (1, 0, 3, 2)),    # <Ai|Bj> = <iA|jB>
    30: (13, 11, "ovvv", (3, 2, 1, 0)),    # <Ab|Ci> = <iC|bA>
    233: (13, 13, "vvvv", (0, 1, 2, 3)),   # <Ab|Cd>
}


def put_hamiltonian(lib, eps, blocks, irr_o, irr_v, fock=None):
    """Write orbital energies and the six integral lists the way the reference's
    intprc does (intprc/clmoio.F).  ``blocks`` maps 'oooo', 'ooov', 'oovv',
    'ovov', 'ovvv', 'vvvv' to dense physicists'-notation arrays <pq|rs>."""
    dpd = DPD(lib, irr_o, irr_v)
    lib.putrec("SCFEVALA", np.asarray(eps, dtype=np.float64))
    if fock is not None:
        lib.putrec("FOCKMAT", np.asarray(fock, dtype=np.float64))
    for lst, (tl, tr, key, perm) in INTEGRAL_LISTS.items():
        dense = blocks[key] if perm == (0, 1, 2, 3) else blocks[key].transpose(perm)
        put_dense_list(lib, dpd, lst, tl, tr, dense)
    return dpd
