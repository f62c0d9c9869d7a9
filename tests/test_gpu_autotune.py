"""GPU tests of the tile autotuner of the tensor-core contractions
(aces_set_autotune).

With the tuner on, the first product of each shape class times the tile
variants that apply to it (one CTA per tile or CTA pairs and split K or not
for single and grouped products, 144- or 256-wide tiles for the batched (T)
launches) and later products of the class reuse the fastest.  Every variant must meet the same bound as the
default (|C - C_fp64| <= 4e-5 (|A||B|)_ij, see test_gpu_split.py), the trial
runs must leave the caller's output exactly as one product would (beta != 0
runs go to a scratch array), a class is tuned once, the CCSD energy stays
within the split path's 1e-6 Eh of the FP64 oracle, and CCSD / (T) energies
match the built-in rules' up to rounding order.  Each test switches the
tuner off again, so the rest of the suite runs the built-in rules.
"""
import pytest

import acesb200 as ab
from oracle.hamiltonian import synthetic
from oracle import ccsd
from test_gpu_ccsd import setup_lists

pytestmark = pytest.mark.gpu


@pytest.fixture
def lib():
    lib = ab.load()
    lib.init(0)
    lib.set_autotune(2)   # forget choices of earlier tests
    lib.set_autotune(1)
    try:
        yield lib
    finally:
        lib.set_autotune(0)
        lib.set_autotune(2)


# (1000, 260, 777): few output tiles, so split K, no split and CTA pairs are
# all candidates; beta != 0 sends the trial runs to scratch.  (300, 2000, 1000)
# with beta = 0 tunes in the output itself.  (70000, 20, 180): many tiles,
# pairs against one CTA per tile.
SHAPES = [(1000, 260, 777, "T", "N", 0.5), (300, 2000, 1000, "T", "N", 0.0),
          (70000, 20, 180, "N", "T", 1.0)]


def _xgemm(lib, m, n, k, ta, tb, beta, seed):
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    A = torch.randn((m, k) if ta == "N" else (k, m), generator=g, dtype=torch.float64)
    B = torch.randn((k, n) if tb == "N" else (n, k), generator=g, dtype=torch.float64)
    A = A * torch.exp(torch.randn(A.shape, generator=g, dtype=torch.float64))
    Cm = torch.randn((m, n), generator=g, dtype=torch.float64)
    opA = A if ta == "N" else A.T
    opB = B if tb == "N" else B.T
    ref = 1.3 * opA @ opB + beta * Cm
    bound = 1.3 * opA.abs() @ opB.abs()
    dA, dB, dC = A.T.contiguous().cuda(), B.T.contiguous().cuda(), Cm.T.contiguous().cuda()
    lib.xgemm(ta, tb, m, n, k, 1.3, dA.data_ptr(), A.shape[0], dB.data_ptr(), B.shape[0], beta,
              dC.data_ptr(), m, precision=ab.PREC_BF16X3)
    err = (dC.cpu().T - ref).abs()
    return (err / (bound + 1e-30)).max().item(), bool((err <= 4e-5 * bound + 1e-12).all())


def test_autotuned_products_meet_the_split_bound_and_tune_once(lib):
    assert lib.autotune_stats() == (0, 0, 0.0)
    for i, (m, n, k, ta, tb, beta) in enumerate(SHAPES):
        before = lib.autotune_stats()[0]
        rel, ok = _xgemm(lib, m, n, k, ta, tb, beta, 31 + i)
        assert ok and rel < 2e-5, (m, n, k, rel)
        classes, changed, ms = lib.autotune_stats()
        assert classes > before, (m, n, k)      # this shape's class was timed
        # the same shape again: served from the cache, same bound
        rel, ok = _xgemm(lib, m, n, k, ta, tb, beta, 131 + i)
        assert ok and rel < 2e-5, (m, n, k, rel)
        assert lib.autotune_stats()[0] == classes
    classes, changed, ms = lib.autotune_stats()
    assert ms > 0.0 and 0 <= changed <= classes
    # mode 2 forgets every choice, mode 0 turns the tuner off
    lib.set_autotune(2)
    assert lib.autotune_stats() == (0, 0, 0.0)
    lib.set_autotune(0)
    rel, ok = _xgemm(lib, *SHAPES[0], 7)
    assert ok and lib.autotune_stats()[0] == 0


def test_autotuned_ccsd_matches_oracle_and_default(lib):
    """Split CCSD with tuned tiles (tuning in the first cycle, the residual
    graph captured on the second replaying the cached variants) against the
    FP64 oracle and against the built-in rules."""
    ham = synthetic(10, 90, 120, seed=2)
    setup_lists(lib, ham)
    tuned = lib.xvcc(cc_conv=8, cc_maxcyc=60, cc_exporder=5, precision=ab.PREC_BF16X3,
                     use_graph=1)
    assert lib.autotune_stats()[0] > 0
    lib.set_autotune(0)
    plain = lib.xvcc(cc_conv=8, cc_maxcyc=60, cc_exporder=5, precision=ab.PREC_BF16X3,
                     use_graph=1)
    ref = ccsd.run_ccsd(ham, cc_conv=8, maxcyc=60, exporder=5)
    assert tuned.converged == 1
    assert abs(tuned.e_ccsd - ref["e_final"]) < 1e-6, tuned.e_ccsd - ref["e_final"]
    assert abs(tuned.e_ccsd - plain.e_ccsd) < 1e-7


def test_autotuned_triples_match_default_tiles(lib):
    """v = 150: the batched (T) class launches (M = v^2, N = v = 150 FP32
    outputs) time the 128 x 256 tile against the 128 x 144 tiles on the first
    batch (the beta = 0 class launch); the energies equal the built-in rule's
    up to FP32 rounding order, as in the wide/narrow test of
    test_gpu_triples.py."""
    ham = synthetic(4, 150, 60, seed=12, bscale=0.5)
    setup_lists(lib, ham)
    tuned = lib.xvcc(cc_conv=9, cc_maxcyc=60, triples=1, precision=ab.PREC_BF16X3)
    classes, changed, ms = lib.autotune_stats()
    assert classes > 0 and ms > 0.0
    lib.set_autotune(0)
    plain = lib.xvcc(cc_conv=9, cc_maxcyc=60, triples=1, precision=ab.PREC_BF16X3)
    assert abs(tuned.e_ccsd - plain.e_ccsd) < 1e-8
    assert abs(tuned.e_t4 - plain.e_t4) < 1e-13 + 1e-8 * abs(plain.e_t4)
    assert abs(tuned.e_st5 - plain.e_st5) < 1e-14 + 1e-8 * abs(plain.e_st5)


def test_saved_choices_reload_without_timing(lib, tmp_path):
    """Choices saved after tuning and loaded into an emptied cache serve the
    same class with no trial runs (no device time added to the stats)."""
    m, n, k, ta, tb, beta = SHAPES[0]
    rel, ok = _xgemm(lib, m, n, k, ta, tb, beta, 41)
    assert ok
    classes, changed, ms = lib.autotune_stats()
    assert classes >= 1 and ms > 0.0
    path = tmp_path / "choices.txt"
    lib.autotune_save(path)
    lib.set_autotune(2)
    lib.autotune_load(path)
    assert lib.autotune_stats() == (classes, changed, 0.0)
    rel, ok = _xgemm(lib, m, n, k, ta, tb, beta, 42)
    assert ok and rel < 2e-5
    assert lib.autotune_stats() == (classes, changed, 0.0)
