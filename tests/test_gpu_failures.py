"""GPU tests of failure detection: every failure is made on the host or by a
bounded device wait that runs out; none faults, traps or hangs the GPU.

* a non-finite integral list -> ACES_ERR_NAN at the first cycle (the
  reference's CC loop has no such check; its equivalent is the
  non-convergence exit of vcc/vcc.F:1439);
* a stalled iteration whose DIIS error vectors underflow to zero -> the
  bordered DIIS system is singular, ACES_ERR_SINGULAR (the reference stops
  in libr/dodiis.F:49 when dgesv reports a zero pivot);
* the tensor-core kernel's producer made to issue no copies (a host-set
  flag) with a 10 ms wait limit -> its consumers' bounded waits run out and
  aces_xgemm returns ACES_ERR_TIMEOUT; the context stays usable and the next
  product is correct.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
import acesb200 as ab
from oracle.hamiltonian import from_fixture
from test_gpu_ccsd import setup_lists

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    lib = ab.load()
    lib.init(0)
    return lib


def test_nan_in_an_integral_list_is_reported(lib):
    ham = from_fixture(os.path.join(GOLDEN, "h2o_dzp_zmat035.npz"))
    setup_lists(lib, ham)
    nr, nc = lib.list_dims(1, 16)
    col = lib.getlst(1, 1, 1, 16)
    col[nr // 2, 0] = np.nan
    lib.putlst(col, 1, 1, 16)
    with pytest.raises(ab.AcesError) as e:
        lib.xvcc(cc_conv=7, cc_maxcyc=20)
    assert e.value.status == -10
    # a clean set of lists afterwards runs normally
    setup_lists(lib, ham)
    assert abs(lib.xvcc(cc_conv=7, cc_maxcyc=50).e_ccsd - (-0.226005606663)) < 1e-10


def test_nan_orbital_energy_is_reported(lib):
    ham = from_fixture(os.path.join(GOLDEN, "h2o_dzp_zmat035.npz"))
    setup_lists(lib, ham)
    eps = ham.eps.copy()
    eps[3] = np.inf
    lib.putrec("SCFEVALA", eps)
    with pytest.raises(ab.AcesError) as e:
        lib.xvcc(cc_conv=7, cc_maxcyc=20)
    assert e.value.status == -10


def test_singular_diis_system_is_reported(lib):
    """DAMP_CC = 1e-300 stalls the iteration: every damped step is below the
    amplitudes' rounding, the error vectors' dot products underflow to zero,
    and at the second cycle the bordered system [[0, -1], [-1, B]] with B = 0
    has a zero pivot, like dgesv's INFO > 0 in libr/dodiis.F."""
    ham = from_fixture(os.path.join(GOLDEN, "h2o_dzp_zmat035.npz"))
    setup_lists(lib, ham)
    with pytest.raises(ab.AcesError) as e:
        lib.xvcc(cc_conv=7, cc_maxcyc=20, damp=1e-300)
    assert e.value.status == -8
    assert "singular" in str(e.value)


def test_tensor_core_wait_limit_reports_timeout(lib):
    import torch
    m, n, k = 256, 256, 512
    g = torch.Generator(device="cpu").manual_seed(3)
    A = torch.randn((k, m), generator=g, dtype=torch.float64)
    B = torch.randn((k, n), generator=g, dtype=torch.float64)
    dA, dB = A.T.contiguous().cuda(), B.T.contiguous().cuda()
    dC = torch.zeros((n, m), dtype=torch.float64, device="cuda")
    lib.init(0)
    lib.set_wait_limit(0.01)
    lib.debug_inject(1)
    try:
        with pytest.raises(ab.AcesError) as e:
            lib.xgemm("T", "N", m, n, k, 1.0, dA.data_ptr(), k, dB.data_ptr(), k, 0.0,
                      dC.data_ptr(), m, precision=ab.PREC_BF16X3)
        assert e.value.status == -11
    finally:
        lib.debug_inject(0)
        lib.set_wait_limit(4.0)
    torch.cuda.synchronize()
    lib.xgemm("T", "N", m, n, k, 1.0, dA.data_ptr(), k, dB.data_ptr(), k, 0.0, dC.data_ptr(), m,
              precision=ab.PREC_BF16X3)
    out = dC.cpu().T
    ref = A.T @ B
    assert ((out - ref).abs() / (A.abs().T @ B.abs())).max().item() < 4e-5
    with pytest.raises(ab.AcesError):
        lib.set_wait_limit(0.0)
