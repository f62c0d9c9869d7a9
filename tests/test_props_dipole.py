"""GPU test of a first-order property (the reference's PROPS=1 run of
test/zmat.026): the electric dipole of H2O/DZP from the engine's CCSD energy
and its unrelaxed one-particle density, against the reference's printed
dipoles (test/OUTPUT/out.zmat.026:762-763, 794-795).

Collected after the other GPU test files (it uses the Lambda and density
entry points of tests/test_gpu_lambda.py)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
import acesb200 as ab
from oracle.hamiltonian import from_fixture
from test_gpu_lambda import gpu_energy

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    lib = ab.load()
    lib.init(0)
    return lib


def test_dipoles_026_engine_relaxed_by_field_and_unrelaxed_density(lib):
    """H2O/DZP of out.zmat.026 (CCSD first-order properties).

    (a) The engine's total CCSD energy in a field along z, with the SCF
    re-solved at each field (orbital-relaxed; the field-dependent lists are
    made on the host by the oracle's finite-field RHF), differentiated by a
    five-point central difference (F = +-1e-3, +-2e-3 a.u.), gives the
    reference's dipole of the relaxed correlated density, Z = 0.8197061290
    (out.zmat.026:795), to 3e-8.
    (b) At fixed orbitals the field only adds F z to the Fock matrix; the
    engine's unrelaxed one-particle density (xlambda + xdens) gives that
    derivative, Tr(D z), to 1e-9 of the finite difference of its own
    energies.  The difference of (a) and (b) is the orbital-relaxation term
    that the reference's D(ai) expansion adds (out.zmat.026:745)."""
    from oracle.hamiltonian import five_point_derivative, scf_in_field
    ham = from_fixture(os.path.join(GOLDEN, "h2o_dzp_zmat026.npz"))
    o, n = ham.nocc, ham.nmo
    z = ham.dipole[2]

    def e_relaxed(field):
        e_scf, hf = scf_in_field(ham, field)
        return e_scf + gpu_energy(lib, hf, hf.fock)

    mu_relaxed = ham.nucdip[2] - five_point_derivative(e_relaxed, 1e-3)
    assert abs(mu_relaxed - 0.8197061290) < 3e-8, mu_relaxed - 0.8197061290

    f0 = ham.fock.copy()
    fd = five_point_derivative(lambda f: gpu_energy(lib, ham, f0 + f * z), 1e-3)
    gpu_energy(lib, ham, f0)
    lib.xlambda(cc_conv=12, cc_maxcyc=200)
    lib.xdens()
    D = lib.getrec("DENSMAT", n * n).reshape(n, n)
    assert abs(np.sum(D * z) - fd) < 1e-9, np.sum(D * z) - fd
    mu_scf = ham.nucdip[2] - 2.0 * np.trace(z[:o, :o])
    mu_unrelaxed = mu_scf - np.sum(D * z)
    # the orbital relaxation moves the dipole by a few 1e-3 a.u. here
    assert 1e-4 < abs(mu_relaxed - mu_unrelaxed) < 5e-2
