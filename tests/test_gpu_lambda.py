"""GPU tests of xlambda_run / xdens_1pdm: the engine's hand-written backward
pass (adjoint replay of the CCSD residual) against the torch-autograd oracle,
and dE/dx = Tr(D h') against a central finite difference (step 1e-4) of the
engine's own CCSD energies with the Fock matrix f + x h'."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
import acesb200 as ab
from acesb200.dpd import get_dense_list
from oracle.hamiltonian import from_fixture, synthetic
from oracle import ccsd, lambda_ad
from test_gpu_ccsd import setup_lists, read_amplitudes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    lib = ab.load()
    lib.init(0)
    return lib


def read_lambda(lib, dpd, o, v):
    l2 = get_dense_list(lib, dpd, 146, 13, 14).transpose(2, 3, 0, 1)
    col = lib.getlst(1, 1, 1, 190)[:, 0]
    idx, sgn, hpq = dpd.table(9)
    l1 = np.zeros((o, v))
    for a in range(v):
        for i in range(o):
            if hpq[a, i] == 0:
                l1[i, a] = col[idx[a, i]]
    return l1, l2


def gpu_energy(lib, ham, fock):
    lib.init(0)
    pop, vrt = ham.pop_vrt()
    lib.sym_init(pop, vrt)
    B = ccsd.Blocks(ham)
    blocks = dict(oooo=B.oooo, ooov=B.ooov, oovv=B.oovv, ovov=B.ovov, ovvv=B.ovvv, vvvv=B.vvvv)
    o = ham.nocc
    ab.put_hamiltonian(lib, np.diag(fock), blocks, ham.irrep[:o], ham.irrep[o:], fock=fock)
    return lib.xvcc(cc_conv=12, cc_maxcyc=200, cc_exporder=8).e_ccsd


@pytest.mark.parametrize("o,v,naux,seed,irreps", [(3, 10, 20, 2, None), (4, 12, 24, 1005, 4)])
def test_lambda_and_density_match_autograd_oracle(lib, o, v, naux, seed, irreps):
    ham = synthetic(o, v, naux, seed, irreps=irreps, bscale=0.5)
    B, dpd = setup_lists(lib, ham)
    lib.xvcc(cc_conv=12, cc_maxcyc=200)
    cl = lib.xlambda(cc_conv=12, cc_maxcyc=200)
    assert cl.converged == 1
    lib.xdens()
    t1, t2 = read_amplitudes(lib, dpd, o, v)
    l1, l2 = read_lambda(lib, dpd, o, v)
    rl1, rl2 = lambda_ad.solve_lambda(B, t1, t2)
    # lists 190/146 hold the reference's multipliers (lambda_ad.lambda_to_reference)
    L1, L2 = lambda_ad.lambda_to_reference(rl1, rl2)
    np.testing.assert_allclose(l1, L1, atol=1e-10)
    np.testing.assert_allclose(l2, L2, atol=1e-10)
    D = lib.getrec("DENSMAT", (o + v) ** 2).reshape(o + v, o + v)
    np.testing.assert_allclose(D, lambda_ad.density(B, t1, t2, rl1, rl2), atol=1e-10)


def test_density_derivative_matches_central_difference(lib):
    ham = synthetic(5, 18, 30, seed=31, bscale=0.5)
    f0 = ham.fock.copy()
    rng = np.random.default_rng(7)
    hp = rng.normal(0, 0.01, f0.shape)
    hp = 0.5 * (hp + hp.T)   # h', a seeded random symmetric matrix with N(0, 0.01^2) entries
    d = 1e-4
    fd = (gpu_energy(lib, ham, f0 + d * hp) - gpu_energy(lib, ham, f0 - d * hp)) / (2 * d)
    # analytic: Lambda + density at the unperturbed Fock matrix
    gpu_energy(lib, ham, f0)
    lib.xlambda(cc_conv=12, cc_maxcyc=200)
    lib.xdens()
    n = f0.shape[0]
    D = lib.getrec("DENSMAT", n * n).reshape(n, n)
    assert abs(np.sum(D * hp) - fd) < 1e-11 + 1e-6 * abs(fd)


def test_lambda_h2o_dzp_symmetry_blocked(lib):
    ham = from_fixture(os.path.join(GOLDEN, "h2o_dzp_zmat026.npz"))
    B, dpd = setup_lists(lib, ham)
    lib.xvcc(cc_conv=10, cc_maxcyc=60)
    assert lib.xlambda(cc_conv=9, cc_maxcyc=60).converged == 1
    lib.xdens()
    t1, t2 = read_amplitudes(lib, dpd, ham.nocc, ham.nvir)
    l1, l2 = read_lambda(lib, dpd, ham.nocc, ham.nvir)
    # the reference's Lambda cycle (pinned to out.zmat.026's xlambda history
    # in tests/test_oracle_lambda.py) converges to the lists' multipliers
    h = ccsd.run_ccsd(ham, cc_conv=10, maxcyc=60, exporder=5)
    r = lambda_ad.iterate_lambda(h["blocks"], h["t1"], h["t2"], cc_conv=9, maxcyc=60)
    assert r["converged"]
    np.testing.assert_allclose(l1, r["L1"], atol=5e-8)
    np.testing.assert_allclose(l2, r["L2"], atol=5e-8)
    # lambda2 is the pair-symmetric multiplier of T2; its norm is of the size of T2's
    assert np.abs(l2 - l2.transpose(1, 0, 3, 2)).max() < 1e-12
    assert 0.5 < np.linalg.norm(l2) / np.linalg.norm(t2) < 2.0
    n = ham.nmo
    D = lib.getrec("DENSMAT", n * n).reshape(n, n)
    # the correlation density moves electrons from occupied to virtual orbitals
    assert np.trace(D[:ham.nocc, :ham.nocc]) < 0 < np.trace(D[ham.nocc:, ham.nocc:])


def test_lambda_split_precision_matches_fp64(lib):
    ham = synthetic(6, 140, 60, seed=41, bscale=0.5)
    setup_lists(lib, ham)
    rng = np.random.default_rng(9)
    hp = rng.normal(0, 0.01, (146, 146))
    hp = 0.5 * (hp + hp.T)
    out = {}
    for prec in (ab.PREC_FP64, ab.PREC_BF16X3):
        lib.xvcc(cc_conv=9, cc_maxcyc=80, precision=prec)
        lib.xlambda(cc_conv=9, cc_maxcyc=80, precision=prec)
        lib.xdens()
        out[prec] = np.sum(lib.getrec("DENSMAT", 146 * 146).reshape(146, 146) * hp)
    assert abs(out[ab.PREC_BF16X3] - out[ab.PREC_FP64]) < 1e-6 * max(1.0, abs(out[ab.PREC_FP64]))
