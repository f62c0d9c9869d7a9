"""GPU tests of the split-precision (BF16x3 on tcgen05) contraction path.

Tolerances: each BF16x3 product carries a relative error below 2^-16 (hi/lo
split of both factors, lo*lo dropped) and the sums are FP32 in TMEM, so an
element of C = A B obeys |C - C_fp64| <= 3e-5 * (|A| |B|)_ij + 1e-6*K*2^-24 ...;
the tests assert |C - C_fp64| <= 4e-5 * (|A| |B|)_ij elementwise.  CCSD
energies must agree with the FP64 oracle to 1e-6 Eh (the target accuracy of
the mixed-precision path)."""
import numpy as np
import pytest

import acesb200 as ab
from oracle.hamiltonian import synthetic
from oracle import ccsd
from test_gpu_ccsd import setup_lists, read_amplitudes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    lib = ab.load()
    lib.init(0)
    return lib


# (1000, 260, 777) takes the split-K path; (2000, 1300, 200) and (70000, 20, 180)
# have more output tiles than SMs, so each persistent CTA walks several tiles
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (128, 128, 64), (37, 53, 29), (300, 200, 513),
                                   (129, 7, 1000), (1000, 260, 777), (2000, 1300, 200),
                                   (70000, 20, 180)])
@pytest.mark.parametrize("ta,tb", [("T", "N"), ("N", "T")])
@pytest.mark.parametrize("beta", [0.5, 0.0, 1.0])
def test_xgemm_bf16x3_error_bound(lib, m, n, k, ta, tb, beta):
    import torch
    g = torch.Generator(device="cpu").manual_seed(m + 11 * n + 101 * k)
    A = torch.randn((m, k) if ta == "N" else (k, m), generator=g, dtype=torch.float64)
    B = torch.randn((k, n) if tb == "N" else (n, k), generator=g, dtype=torch.float64)
    # spread magnitudes over a few decades like CC intermediates
    A = A * torch.exp(torch.randn(A.shape, generator=g, dtype=torch.float64))
    Cm = torch.randn((m, n), generator=g, dtype=torch.float64)
    opA = A if ta == "N" else A.T
    opB = B if tb == "N" else B.T
    ref = 1.3 * opA @ opB + beta * Cm
    bound = 1.3 * opA.abs() @ opB.abs()
    dA = A.T.contiguous().cuda()
    dB = B.T.contiguous().cuda()
    dC = Cm.T.contiguous().cuda()
    lib.xgemm(ta, tb, m, n, k, 1.3, dA.data_ptr(), A.shape[0], dB.data_ptr(), B.shape[0], beta,
              dC.data_ptr(), m, precision=ab.PREC_BF16X3)
    out = dC.cpu().T
    err = (out - ref).abs()
    assert torch.all(err <= 4e-5 * bound + 1e-12), (err / (bound + 1e-30)).max().item()
    # and it is a genuine split: much closer than a single BF16 product would be
    assert (err / (bound + 1e-30)).max().item() < 2e-5


# Long contractions: the FP32 accumulation chunk shortens with K (512 K
# elements up to K = 36864, 256 up to 73728, 128 beyond), the lengths of the
# particle-particle contractions at o = 30, v = 270 (K = v^2 = 72900).  These
# two shapes run the 256- and 128-element chunks (with split K: 4 output tiles).
@pytest.mark.parametrize("k", [40000, 80000])
@pytest.mark.parametrize("ta,tb", [("T", "N"), ("N", "T")])
def test_xgemm_bf16x3_long_k_chunks(lib, k, ta, tb):
    import torch
    m = n = 256
    g = torch.Generator(device="cpu").manual_seed(k + (ta == "T"))
    A = torch.randn((m, k) if ta == "N" else (k, m), generator=g, dtype=torch.float64)
    B = torch.randn((k, n) if tb == "N" else (n, k), generator=g, dtype=torch.float64)
    A = A * torch.exp(torch.randn(A.shape, generator=g, dtype=torch.float64))
    Cm = torch.randn((m, n), generator=g, dtype=torch.float64)
    opA = A if ta == "N" else A.T
    opB = B if tb == "N" else B.T
    ref = 0.8 * opA @ opB + 1.0 * Cm
    bound = 0.8 * opA.abs() @ opB.abs()
    dA = A.T.contiguous().cuda()
    dB = B.T.contiguous().cuda()
    dC = Cm.T.contiguous().cuda()
    lib.xgemm(ta, tb, m, n, k, 0.8, dA.data_ptr(), A.shape[0], dB.data_ptr(), B.shape[0], 1.0,
              dC.data_ptr(), m, precision=ab.PREC_BF16X3)
    out = dC.cpu().T
    err = (out - ref).abs()
    assert torch.all(err <= 4e-5 * bound + 1e-12), (err / (bound + 1e-30)).max().item()
    # the FP32 partial sums of a chunk do not drift: the error relative to the
    # bound stays at the size of a single split product's
    assert (err / (bound + 1e-30)).max().item() < 2e-5


def test_ccsd_bf16x3_energy_within_1e6(lib):
    ham = synthetic(10, 90, 120, seed=2)
    setup_lists(lib, ham)
    cfg = lib.xvcc(cc_conv=8, cc_maxcyc=60, cc_exporder=5, precision=ab.PREC_BF16X3)
    ref = ccsd.run_ccsd(ham, cc_conv=8, maxcyc=60, exporder=5)
    assert cfg.converged == 1
    assert abs(cfg.e_ccsd - ref["e_final"]) < 1e-6, cfg.e_ccsd - ref["e_final"]


def test_ccsd_bf16x3_then_fp64_same_lists(lib):
    """FP64 and split runs read the same lists; the FP64 run is exact to the oracle."""
    ham = synthetic(8, 64, 90, seed=4)
    setup_lists(lib, ham)
    split = lib.xvcc(cc_conv=8, cc_maxcyc=60, precision=ab.PREC_BF16X3).e_ccsd
    exact = lib.xvcc(cc_conv=8, cc_maxcyc=60, precision=ab.PREC_FP64).e_ccsd
    ref = ccsd.run_ccsd(ham, cc_conv=8, maxcyc=60)["e_final"]
    assert abs(exact - ref) < 1e-11
    assert abs(split - ref) < 1e-6


# The CTA-pair tile variant (aces_set_tc_pairs(1): tcgen05 cta_group::2 on
# 256 x 128 tiles for products of >= 256 rows) obeys the same bound.  Shapes:
# ragged rows in the second CTA of a pair (300), split K (1000 x 260 x 777),
# several pair tiles per CTA pair (2000 x 1300), a thin ragged N = 20 whose
# B half per CTA is 16 rows, and multi-chunk K.
@pytest.mark.parametrize("m,n,k", [(300, 200, 513), (1000, 260, 777), (2000, 1300, 200),
                                   (70000, 20, 180), (256, 256, 40000)])
@pytest.mark.parametrize("beta", [0.0, 1.0])
def test_xgemm_bf16x3_pairs_error_bound(lib, m, n, k, beta):
    import torch
    g = torch.Generator(device="cpu").manual_seed(7 * m + n + k)
    A = torch.randn((k, m), generator=g, dtype=torch.float64)
    B = torch.randn((k, n), generator=g, dtype=torch.float64)
    A = A * torch.exp(torch.randn(A.shape, generator=g, dtype=torch.float64))
    Cm = torch.randn((m, n), generator=g, dtype=torch.float64)
    ref = 1.1 * A.T @ B + beta * Cm
    bound = 1.1 * A.T.abs() @ B.abs()
    dA = A.T.contiguous().cuda()   # column-major (k x m) A: op(A) = A^T
    dB = B.T.contiguous().cuda()
    dC = Cm.T.contiguous().cuda()
    lib.set_tc_pairs(1)
    try:
        lib.xgemm("T", "N", m, n, k, 1.1, dA.data_ptr(), k, dB.data_ptr(), k, beta,
                  dC.data_ptr(), m, precision=ab.PREC_BF16X3)
    finally:
        lib.set_tc_pairs(0)
    out = dC.cpu().T
    err = (out - ref).abs()
    assert torch.all(err <= 4e-5 * bound + 1e-12), (err / (bound + 1e-30)).max().item()
    assert (err / (bound + 1e-30)).max().item() < 2e-5


def test_ccsd_bf16x3_pairs_energy_within_1e6(lib):
    """A split CCSD whose ladder, ring and (T)-free contractions run on CTA pairs."""
    ham = synthetic(10, 90, 120, seed=2)
    setup_lists(lib, ham)
    lib.set_tc_pairs(1)
    try:
        cfg = lib.xvcc(cc_conv=8, cc_maxcyc=60, cc_exporder=5, precision=ab.PREC_BF16X3)
    finally:
        lib.set_tc_pairs(0)
    ref = ccsd.run_ccsd(ham, cc_conv=8, maxcyc=60, exporder=5)
    assert cfg.converged == 1
    assert abs(cfg.e_ccsd - ref["e_final"]) < 1e-6, cfg.e_ccsd - ref["e_final"]
