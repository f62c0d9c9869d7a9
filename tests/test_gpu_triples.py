"""GPU tests of the (T) correction against the oracle and the reference's
golden energies (test/OUTPUT/out.zmat.020:665-688)."""
import os

import pytest

from conftest import GOLDEN
import acesb200 as ab
from oracle.hamiltonian import from_fixture, synthetic
from oracle import ccsd
from oracle.triples import triples
from test_gpu_ccsd import setup_lists

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    lib = ab.load()
    lib.init(0)
    return lib


def test_ccsd_t_h2o_dzp_matches_reference(lib):
    ham = from_fixture(os.path.join(GOLDEN, "h2o_dzp_zmat020.npz"))
    setup_lists(lib, ham)
    cfg = lib.xvcc(cc_conv=7, cc_maxcyc=50, cc_exporder=5, triples=1)
    # out.zmat.020:679-680, 688
    assert abs(cfg.e_t4 - (-0.003870011955)) < 2e-11
    assert abs(cfg.e_st5 - 0.000163057248) < 2e-11
    assert abs(ham.e_scf + cfg.e_ccsd + cfg.e_t4 + cfg.e_st5 - (-76.273476801298)) < 1e-10
    assert abs(lib.getrec("E4T", 1)[0] - cfg.e_t4) == 0.0


@pytest.mark.parametrize("o,v,naux,seed,irreps", [(5, 23, 40, 8, None), (6, 30, 48, 1004, 8)])
def test_triples_matches_oracle(lib, o, v, naux, seed, irreps):
    ham = synthetic(o, v, naux, seed, irreps=irreps)
    setup_lists(lib, ham)
    cfg = lib.xvcc(cc_conv=10, cc_maxcyc=80, cc_exporder=5, triples=1)
    ref = ccsd.run_ccsd(ham, cc_conv=10, maxcyc=80, exporder=5)
    e4, e5 = triples(ham, ref["t1"], ref["t2"])
    assert abs(cfg.e_t4 - e4) < 1e-12 + 1e-9 * abs(e4)
    assert abs(cfg.e_st5 - e5) < 1e-12 + 1e-9 * abs(e5)


def test_triples_split_matches_fp64(lib):
    """v >= 128 engages the tcgen05 BF16x3 contractions of W."""
    ham = synthetic(4, 136, 60, seed=12, bscale=0.5)
    setup_lists(lib, ham)
    exact = lib.xvcc(cc_conv=9, cc_maxcyc=60, triples=1, precision=ab.PREC_FP64)
    split = lib.xvcc(cc_conv=9, cc_maxcyc=60, triples=1, precision=ab.PREC_BF16X3)
    assert abs(split.e_ccsd - exact.e_ccsd) < 1e-7
    assert abs(split.e_t4 - exact.e_t4) < 1e-8 + 1e-6 * abs(exact.e_t4)
    assert abs(split.e_st5 - exact.e_st5) < 1e-9 + 1e-6 * abs(exact.e_st5)


def test_triples_wide_tiles_match_narrow_tiles(lib):
    """The (T) class launches on 128 x 256 tiles (aces_set_tc_wide(1), the
    default for single-chunk FP32 output with 144 < N <= 256) against the
    144-wide tiles: v = 160 puts classes a/b (N = 160) and the transposed
    class c (N = c = 160) on one wide tile each, where the narrow tiles split
    N into 144 + 16; the W sums differ only in FP32 rounding order."""
    ham = synthetic(4, 160, 60, seed=12, bscale=0.5)
    setup_lists(lib, ham)
    wide = lib.xvcc(cc_conv=9, cc_maxcyc=60, triples=1, precision=ab.PREC_BF16X3)
    lib.set_tc_wide(0)
    try:
        narrow = lib.xvcc(cc_conv=9, cc_maxcyc=60, triples=1, precision=ab.PREC_BF16X3)
    finally:
        lib.set_tc_wide(1)
    assert wide.e_ccsd == narrow.e_ccsd
    assert abs(wide.e_t4 - narrow.e_t4) < 1e-14 + 1e-9 * abs(narrow.e_t4)
    assert abs(wide.e_st5 - narrow.e_st5) < 1e-15 + 1e-9 * abs(narrow.e_st5)


@pytest.mark.parametrize("prec", [ab.PREC_FP64, ab.PREC_BF16X3])
def test_triplet_shards_add_up_to_the_full_triples(lib, prec):
    """The per-GPU (T) shards (triples_rank / triples_nranks), evaluated here one
    after another on one GPU, sum to the unsharded energies; their union is
    checked against the oracle's unique-triplet sum of the same shards."""
    from acesb200.parallel import triplet_shard
    from oracle.triples import triples_unique
    ham = synthetic(5, 130, 48, seed=21, bscale=0.5)
    setup_lists(lib, ham)
    full = lib.xvcc(cc_conv=9, cc_maxcyc=60, triples=1, precision=prec)
    for nranks in (2, 3):
        e4 = e5 = 0.0
        for r in range(nranks):
            c = lib.xvcc(cc_conv=9, cc_maxcyc=60, triples=1, precision=prec, triples_rank=r,
                         triples_nranks=nranks)
            e4 += c.e_t4
            e5 += c.e_st5
        assert abs(e4 - full.e_t4) < 1e-13 + 1e-11 * abs(full.e_t4)
        assert abs(e5 - full.e_st5) < 1e-14 + 1e-11 * abs(full.e_st5)
    if prec == ab.PREC_FP64:
        small = synthetic(4, 12, 20, seed=22)
        setup_lists(lib, small)
        ref = ccsd.run_ccsd(small, cc_conv=10, maxcyc=80, exporder=5)
        s4, s5 = triples_unique(small, ref["t1"], ref["t2"], triplet_shard(4, 1, 3))
        c = lib.xvcc(cc_conv=10, cc_maxcyc=80, triples=1, precision=prec, triples_rank=1,
                     triples_nranks=3)
        assert abs(c.e_t4 - s4) < 1e-12 + 1e-9 * abs(s4)
        assert abs(c.e_st5 - s5) < 1e-13 + 1e-9 * abs(s5)
    with pytest.raises(ab.AcesError):
        lib.xvcc(cc_conv=9, cc_maxcyc=60, triples=1, precision=prec, triples_rank=3,
                 triples_nranks=3)
