"""CPU tests: the Lambda/density oracle (torch autograd on the restated CCSD
residual) reproduces finite differences of the CCSD energy."""
import numpy as np
import pytest

from oracle.hamiltonian import synthetic
from oracle import ccsd, lambda_ad


def _energy_with(hp, x, **kw):
    ham = synthetic(3, 8, 16, seed=2, bscale=0.5)
    ham.fock = ham.fock + x * hp
    return ccsd.run_ccsd(ham, cc_conv=13, maxcyc=300)["e_final"]


def test_density_trace_equals_central_difference():
    ham = synthetic(3, 8, 16, seed=2, bscale=0.5)
    h = ccsd.run_ccsd(ham, cc_conv=13, maxcyc=300)
    B, t1, t2 = h["blocks"], h["t1"], h["t2"]
    l1, l2 = lambda_ad.solve_lambda(B, t1, t2)
    assert np.abs(l2 - l2.transpose(1, 0, 3, 2)).max() < 1e-14
    D = lambda_ad.density(B, t1, t2, l1, l2)
    rng = np.random.default_rng(0)
    hp = rng.normal(0, 0.01, (11, 11))
    hp = 0.5 * (hp + hp.T)
    d = 1e-4   # the central-difference step of the Lambda/density workload
    fd = (_energy_with(hp, d) - _energy_with(hp, -d)) / (2 * d)
    assert abs(fd - np.sum(D * hp)) < 1e-12 + 1e-5 * abs(fd)


def test_lambda_full_space_and_subspace_give_same_gradient():
    ham = synthetic(3, 7, 14, seed=5, bscale=0.5)
    h = ccsd.run_ccsd(ham, cc_conv=13, maxcyc=300)
    B, t1, t2 = h["blocks"], h["t1"], h["t2"]
    Ds = lambda_ad.density(B, t1, t2, *lambda_ad.solve_lambda(B, t1, t2, symmetric=True))
    Df = lambda_ad.density(B, t1, t2, *lambda_ad.solve_lambda(B, t1, t2, symmetric=False))
    hp = np.random.default_rng(3).normal(0, 0.01, Ds.shape)
    hp = hp + hp.T
    assert abs(np.sum(Ds * hp) - np.sum(Df * hp)) < 1e-12


# out.zmat.026:704-722 (xlambda after the CCSD of H2O/DZP, R=0.96 A, A=104 deg):
# largest element of the change and of the DIIS residual in each of the 9 cycles
GOLD_026_LAMBDA_RES = [0.39693849e-02, 0.33716283e-03, 0.28630025e-03, 0.89593700e-04,
                       0.36071913e-04, 0.83980005e-05, 0.22057665e-05, 0.25170668e-06,
                       0.58687065e-07]
GOLD_026_LAMBDA_DRES = [0.39693849e-02, 0.33853268e-03, 0.21420212e-03, 0.42868084e-04,
                        0.18635215e-04, 0.24425820e-05, 0.81159251e-06, 0.12641625e-06,
                        0.57497931e-07]


def test_lambda_iterations_match_reference():
    """The reference's Lambda cycle (initial multipliers = T, NEWT2 update,
    DIIS over its own L1/L2 vector) reproduces every cycle of xlambda in
    out.zmat.026 -- which pins the multiplier convention: the reference's
    L1, L2 map to the Lagrange multipliers of the spin-adapted residual as
    l1 = 2 L1, l2 = 2 L2 - L2~ (lambda_ad.lambda_to_reference)."""
    import os
    from conftest import GOLDEN
    from oracle.hamiltonian import from_fixture
    ham = from_fixture(os.path.join(GOLDEN, "h2o_dzp_zmat026.npz"))
    h = ccsd.run_ccsd(ham, cc_conv=7, maxcyc=50, exporder=5)
    r = lambda_ad.iterate_lambda(h["blocks"], h["t1"], h["t2"], cc_conv=7, maxcyc=50, exporder=5)
    assert r["converged"] and r["ncycle"] == 9
    # magnitudes: the sign of the largest element depends on the MO phases.
    # Agreement is ~1e-5 relative per cycle (1e-7 for the CCSD cycles): the
    # first cycle, before any DIIS step, agrees to 3e-6 (7e-7 when Lambda
    # starts from the amplitudes of one more update); another multiplier
    # convention or initial guess moves the first cycle by 27 % to a factor 6.
    np.testing.assert_allclose(np.abs(r["res"]), GOLD_026_LAMBDA_RES, rtol=3e-5)
    np.testing.assert_allclose(np.abs(r["dres"]), GOLD_026_LAMBDA_DRES, rtol=3e-5)
    L1, L2 = lambda_ad.lambda_to_reference(r["l1"], r["l2"])
    np.testing.assert_allclose(L1, r["L1"], atol=1e-15)
    np.testing.assert_allclose(L2, r["L2"], atol=1e-15)
