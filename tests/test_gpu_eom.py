"""GPU tests of xvee_run (singlet EOM-EE-CCSD, PROGRAM VEE,
vee/doeomee_david.F): the engine's Davidson on its transposed-Jacobian
products (the reverse replay of the residual pass) against

* the reference's golden roots of out.zmat.035.ccsd (H2O/DZP, one root per
  C2v irrep; the reference converges them to about 1e-7 Eh);
* the oracle's Davidson (torch autograd products) on a synthetic 8-irrep
  system, two roots in two irreps, to the Davidson tolerance.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
import acesb200 as ab
from oracle.hamiltonian import from_fixture, synthetic
from oracle import ccsd, eom
from test_gpu_ccsd import setup_lists
from test_oracle_eom import GOLD_OMEGA

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    lib = ab.load()
    lib.init(0)
    return lib


@pytest.mark.parametrize("prec", [ab.PREC_FP64, ab.PREC_BF16X3])
def test_eom_h2o_dzp_matches_reference(lib, prec):
    ham = from_fixture(os.path.join(GOLDEN, "h2o_dzp_zmat035.npz"))
    setup_lists(lib, ham)
    lib.xvcc(cc_conv=10, cc_maxcyc=60, cc_exporder=5, precision=prec)
    cfg, w = lib.xvee([1, 1, 1, 1], eom_conv=8, eom_maxcyc=60, precision=prec)
    assert all(cfg.converged[h] for h in range(4))
    for h in range(4):
        assert abs(w[h][0] - GOLD_OMEGA[h]) < 1e-7, (h, w[h][0], GOLD_OMEGA[h])
    rec = lib.getrec("EOMEXCIT", 64).reshape(8, 8)
    np.testing.assert_array_equal(rec[:4, 0], [w[h][0] for h in range(4)])


def test_eom_synthetic_irreps_match_oracle(lib):
    ham = synthetic(4, 14, 30, seed=1002, irreps=8, bscale=0.5)
    setup_lists(lib, ham)
    lib.xvcc(cc_conv=10, cc_maxcyc=80, cc_exporder=5)
    ref_cc = ccsd.run_ccsd(ham, cc_conv=10, maxcyc=80, exporder=5)
    irr = np.asarray(ham.irrep)
    # two irreps with enough single excitations for two roots each
    counts = [int(np.sum((irr[:4, None] ^ irr[None, 4:]) == h)) for h in range(8)]
    hs = [h for h in range(8) if counts[h] >= 4][:2]
    nroots = [2 if h in hs else 0 for h in range(8)]
    ref = eom.eom_ccsd(ham, ref_cc["t1"], ref_cc["t2"], nroots, tol=1e-9)
    cfg, w = lib.xvee(nroots, eom_conv=9, eom_maxcyc=80)
    for h in hs:
        np.testing.assert_allclose(w[h], ref[h], rtol=0, atol=1e-8)
    with pytest.raises(ab.AcesError):
        lib.xvee([9], eom_conv=8)
