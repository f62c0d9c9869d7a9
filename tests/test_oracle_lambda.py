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
