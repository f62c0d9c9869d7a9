"""CPU tests: the oracle pinned to the reference's golden regression outputs.

Golden values are quoted from the reference's captured outputs:
  test/OUTPUT/out.zmat.035.ccsd (H2O/DZP CCSD, R=0.957 A, A=104.5 deg):
    SCF energy :443, MP2 pieces FORMT2 block, per-iteration CCSD energies and
    residual maxima :555-650;
  test/OUTPUT/out.zmat.020 (H2O/DZP CCSD(T), R=1.0 A, A=104 deg): :650-688.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle.hamiltonian import from_fixture, synthetic
from oracle import ccsd, ccsd_so
from oracle.triples import triples

# out.zmat.035.ccsd: "Summary of iterative solution of CC equations"
GOLD_035_ITER = [
    -0.216941906555, -0.221394755280, -0.224859749997, -0.225631953135, -0.225982984496,
    -0.226003683353, -0.226005732666, -0.226005537711, -0.226005607150, -0.226005622312,
    -0.226005608912,
]
GOLD_035_FINAL = -0.226005606663
# |largest element of residual vector| / |DIIS residual| per iteration
GOLD_035_RES = [0.80606944e-02, 0.22937753e-02, 0.10929478e-02, 0.16750983e-03,
                0.12812421e-03, 0.43273349e-04, 0.16675441e-04, 0.24354994e-05,
                0.38904255e-06, 0.10076627e-06, 0.16830056e-07]
GOLD_035_DRES = [0.80606944e-02, 0.24718504e-02, 0.86146781e-03, 0.86891628e-04,
                 0.82442868e-04, 0.17998710e-04, 0.49789397e-05, 0.79920082e-06,
                 0.24698868e-06, 0.61904624e-07, 0.10316917e-07]


# out.zmat.026 (H2O/DZP, R=0.96 A, A=104 deg, the CCSD of the first-order
# properties job): "Summary of iterative solution of CC equations" :665-677,
# per-iteration maxima :570-632, amplitude norms :646/:658, MP2 :530-545
GOLD_026_ITER = [
    -0.217208070842, -0.221613733226, -0.225105466772, -0.225882139977, -0.226238701153,
    -0.226259784917, -0.226261880533, -0.226261678232, -0.226261750159, -0.226261766032,
    -0.226261752235, -0.226261749882,
]
GOLD_026_RES = [0.81020837e-02, 0.23343131e-02, 0.11138743e-02, 0.17013937e-03,
                0.13042336e-03, 0.43938616e-04, 0.16929190e-04, 0.24720746e-05,
                0.39616913e-06, 0.10378036e-06, 0.17358044e-07]
GOLD_026_DRES = [0.81020837e-02, 0.25114774e-02, 0.87657768e-03, 0.88183039e-04,
                 0.83485227e-04, 0.18278810e-04, 0.50242777e-05, 0.82730424e-06,
                 0.25734839e-06, 0.62318640e-07, 0.10602429e-07]


@pytest.fixture(scope="module")
def h2o035():
    return from_fixture(os.path.join(GOLDEN, "h2o_dzp_zmat035.npz"))


@pytest.fixture(scope="module")
def h2o020():
    return from_fixture(os.path.join(GOLDEN, "h2o_dzp_zmat020.npz"))


def test_scf_fixture_matches_reference(h2o035, h2o020):
    # SCFENEG / NUCREP records of test/zmat.035.ccsd and test/zmat.020 TEST.DAT
    assert abs(h2o035.e_scf - (-76.0465033211)) < 1e-10
    assert abs(h2o035.e_nuc - 9.19693438045) < 1e-10
    assert abs(h2o020.e_scf - (-76.0407105174)) < 1e-10
    # orbital eigenvalues, out.zmat.035.ccsd orbital table (energy order)
    e = np.sort(h2o035.eps)
    gold = [-20.5576668354, -1.3457606900, -0.7109542608, -0.5756658799, -0.5027612661,
            0.2261806614, 0.3179986035, 0.8454784062, 48.0327497683]
    np.testing.assert_allclose(e[[0, 1, 2, 3, 4, 5, 6, 7, 25]], gold, atol=2e-9)
    pop, vrt = h2o035.pop_vrt()
    assert list(pop) == [3, 1, 1, 0] and list(vrt) == [10, 3, 6, 2]


def test_mp2_matches_reference(h2o035):
    B = ccsd.Blocks(h2o035)
    t1, t2 = ccsd.mp2_guess(B)
    eaa, eab, etot = ccsd.energy(B, t1, t2)
    # FORMT2 block of out.zmat.035.ccsd: E2(AA), E2(AB), E2(TOT)
    assert abs(eaa - (-0.025966426160)) < 1e-10
    assert abs(eab - (-0.165009054236)) < 1e-10
    assert abs(etot - (-0.216941906555)) < 1e-10
    # "Norm of T2AB vector (3087 symmetry allowed elements): 0.1983570155"
    assert abs(np.linalg.norm(t2) - 0.1983570155) < 1e-9
    assert np.count_nonzero(np.abs(B.oovv) > 1e-14) <= 3087


def test_ccsd_iterations_match_reference(h2o035):
    h = ccsd.run_ccsd(h2o035, cc_conv=7, maxcyc=50, exporder=5)
    assert h["converged"] and h["ncycle"] == 11
    np.testing.assert_allclose(h["energies"], GOLD_035_ITER + [h["energies"][-1]], atol=1e-10)
    # magnitudes only: the sign of an amplitude depends on the MO phase convention
    np.testing.assert_allclose(np.abs(h["res"]), GOLD_035_RES, rtol=2e-7)
    np.testing.assert_allclose(np.abs(h["dres"]), GOLD_035_DRES, rtol=2e-7)
    assert abs(h["e_final"] - GOLD_035_FINAL) < 1e-10
    # "Norm of T1AA vector (39 ...): 0.0191689919", "Norm of T2AB vector ...: 0.2195553160"
    assert abs(np.linalg.norm(h["t1"]) - 0.0191689919) < 1e-9
    assert abs(np.linalg.norm(h["t2"]) - 0.2195553160) < 1e-9


def test_ccsd_t_matches_reference(h2o020):
    h = ccsd.run_ccsd(h2o020, cc_conv=7, maxcyc=50, exporder=5)
    # out.zmat.020:650 CCSD total, :679-680 E[4]T / E[5]ST, :688 CCSD(T)
    assert abs(h["e_final"] + h2o020.e_scf - (-76.269769846591)) < 1e-10
    e4, e5 = triples(h2o020, h["t1"], h["t2"])
    assert abs(e4 - (-0.003870011955)) < 2e-11
    assert abs(e5 - 0.000163057248) < 2e-11
    assert abs(h["e_final"] + h2o020.e_scf + e4 + e5 - (-76.273476801298)) < 1e-10


def test_closed_shell_equals_spin_orbital_nonhf():
    ham = synthetic(3, 5, 12, seed=7)
    rng = np.random.default_rng(1)
    h = rng.normal(0, 0.05, (8, 8))
    ham.fock = ham.fock + h + h.T
    B = ccsd.Blocks(ham)
    t1 = rng.normal(0, 0.05, (3, 5))
    t2 = ccsd.symmetrize_t2(rng.normal(0, 0.05, (3, 3, 5, 5)))
    Z1, Z2 = ccsd.residual(B, t1, t2)
    asym, f, no = ccsd_so.spin_hamiltonian(ham)
    T1, T2 = ccsd_so.to_spin_amplitudes(t1, t2)
    S1, S2 = ccsd_so.residual(asym, f, no, T1, T2)
    np.testing.assert_allclose(S1[0::2, 0::2], Z1, atol=1e-14)
    np.testing.assert_allclose(S2[0::2, 1::2, 0::2, 1::2], Z2, atol=1e-14)
    assert abs(ccsd.energy(B, t1, t2)[2] - ccsd_so.energy(asym, f, no, T1, T2)) < 1e-14


def test_triples_equals_spin_orbital():
    ham = synthetic(3, 6, 14, seed=3)
    h = ccsd.run_ccsd(ham, cc_conv=10)
    t1, t2 = h["t1"], h["t2"]
    asym, f, no = ccsd_so.spin_hamiltonian(ham)
    T1, T2 = ccsd_so.to_spin_amplitudes(t1, t2)
    o = slice(0, no)
    v = slice(no, asym.shape[0])
    eo, ev = np.diag(f)[o], np.diag(f)[v]
    D = (eo[:, None, None, None, None, None] + eo[None, :, None, None, None, None]
         + eo[None, None, :, None, None, None] - ev[None, None, None, :, None, None]
         - ev[None, None, None, None, :, None] - ev[None, None, None, None, None, :])
    X = (np.einsum("jkae,eibc->ijkabc", T2, asym[v, o, v, v])
         - np.einsum("imbc,majk->ijkabc", T2, asym[o, v, o, o]))
    Pi = lambda x: x - x.transpose(1, 0, 2, 3, 4, 5) - x.transpose(2, 1, 0, 3, 4, 5)
    Pa = lambda x: x - x.transpose(0, 1, 2, 4, 3, 5) - x.transpose(0, 1, 2, 5, 4, 3)
    t3c = Pa(Pi(X)) / D
    t3d = Pa(Pi(np.einsum("ia,jkbc->ijkabc", T1, asym[o, o, v, v]))) / D
    e4, e5 = triples(ham, t1, t2)
    assert abs(e4 - np.sum(t3c * D * t3c) / 36) < 1e-16
    assert abs(e5 - np.sum(t3c * D * t3d) / 36) < 1e-18


def test_packed_ladder_equals_dense_ladder(h2o035):
    """The a<=b packed particle-particle ladder (vcc/ladab1.F:55-64) in the
    symmetric/antisymmetric form the engine runs equals the dense
    sum_ef <ab|ef> tau(ij,ef), on the real H2O/DZP integrals at the MP2
    amplitudes and on a synthetic DF system with T1 in tau."""
    B = ccsd.Blocks(h2o035)
    t1, t2 = ccsd.mp2_guess(B)
    tt = ccsd.tau(t1, t2)
    dense = np.einsum("ijef,abef->ijab", tt, B.vvvv, optimize=True)
    np.testing.assert_allclose(ccsd.ladder_packed(B.vvvv, tt), dense, rtol=0, atol=1e-14)
    ham = synthetic(4, 13, 30, seed=9)
    Bs = ccsd.Blocks(ham)
    rng = np.random.default_rng(3)
    t1 = rng.normal(0.0, 0.05, (4, 13))
    t2 = rng.normal(0.0, 0.05, (4, 4, 13, 13))
    t2 = 0.5 * (t2 + t2.transpose(1, 0, 3, 2))
    tt = ccsd.tau(t1, t2)
    dense = np.einsum("ijef,abef->ijab", tt, Bs.vvvv, optimize=True)
    np.testing.assert_allclose(ccsd.ladder_packed(Bs.vvvv, tt), dense,
                               rtol=0, atol=1e-13 * np.abs(dense).max())


def test_ccsd_026_matches_reference():
    """A third geometry (out.zmat.026): SCF, MP2, every CCSD iteration's energy
    and residual maxima, the converged energy and amplitude norms."""
    ham = from_fixture(os.path.join(GOLDEN, "h2o_dzp_zmat026.npz"))
    # E(SCF) :451, nuclear repulsion 9.16938 a.u. (z-matrix analysis)
    assert abs(ham.e_scf - (-76.0462837076)) < 1e-10
    B = ccsd.Blocks(ham)
    t1, t2 = ccsd.mp2_guess(B)
    eaa, eab, etot = ccsd.energy(B, t1, t2)
    assert abs(eaa - (-0.025991950000)) < 1e-10 and abs(eab - (-0.165224170842)) < 1e-10
    assert abs(np.linalg.norm(t2) - 0.1987656990) < 1e-9
    h = ccsd.run_ccsd(ham, cc_conv=7, maxcyc=50, exporder=5)
    assert h["converged"] and h["ncycle"] == 11
    np.testing.assert_allclose(h["energies"], GOLD_026_ITER, atol=1e-10)
    np.testing.assert_allclose(np.abs(h["res"]), GOLD_026_RES, rtol=2e-7)
    np.testing.assert_allclose(np.abs(h["dres"]), GOLD_026_DRES, rtol=2e-7)
    assert abs(h["e_final"] - (-0.226261749882)) < 1e-10
    assert abs(np.linalg.norm(h["t1"]) - 0.0193257962) < 1e-9
    assert abs(np.linalg.norm(h["t2"]) - 0.2200706819) < 1e-9


def test_ccsd_046_config1_geometry_matches_reference():
    """The benchmark geometry (R = 0.9572 A, A = 104.52 deg) in the reference's
    DZP basis with Cartesian d: test/zmat.046 runs it as a UHF-CCSD, whose
    closed-shell solution is the RHF one.  Pinned: nuclear repulsion and SCF
    (out.zmat.046:339,605), MP2 pieces and T2AB norm (:604-608,638), the first
    CC iteration (the same Jacobi step from MP2 in either spin formalism:
    energy and largest residual element, :685-691) and the converged CCSD
    energy (:745; the reference stops at a residual of 1.9e-8, so 5e-9 Eh).
    Iterations 2 onwards differ by design: the UHF DIIS vector weights the
    spin blocks differently from the RHF one (vcc/dodiis0.F)."""
    ham = from_fixture(os.path.join(GOLDEN, "h2o_dzp_zmat046.npz"))
    assert abs(ham.e_nuc - 9.1949465922) < 1e-9
    assert abs(ham.e_scf - (-76.046493464757)) < 2e-10
    B = ccsd.Blocks(ham)
    t1, t2 = ccsd.mp2_guess(B)
    eaa, eab, etot = ccsd.energy(B, t1, t2)
    assert abs(eaa - (-0.025967355589)) < 1e-10 and abs(eab - (-0.165019405916)) < 1e-10
    assert abs(etot - (-0.216954117095)) < 1e-10
    assert abs(np.linalg.norm(t2) - 0.1983798481) < 1e-9
    h = ccsd.run_ccsd(ham, cc_conv=10, maxcyc=60, exporder=5)
    assert h["converged"]
    assert abs(h["energies"][1] - (-0.221404651273)) < 1e-10
    assert abs(abs(h["res"][0]) - 0.80627031e-02) < 2e-7 * 0.80627031e-02
    assert abs(h["e_final"] - (-0.226017627669)) < 5e-9


def test_ccpvdz_config1_fixture():
    """Config 1 (H2O, 0.9572 A / 104.52 deg, cc-pVDZ with spherical d): 24
    basis functions, 5 occupied / 19 virtual, C2v populations; the oracle's
    CCSD converges to max|dT| < 1e-10.  No reference output exists for this
    basis; the fixture's SCF is checked for self-consistency (occupied orbitals
    below the virtual ones, Brillouin: the converged Fock matrix is diagonal)."""
    ham = from_fixture(os.path.join(GOLDEN, "h2o_ccpvdz.npz"))
    assert ham.nmo == 24 and ham.nocc == 5 and ham.nvir == 19
    pop, vrt = ham.pop_vrt()
    assert list(pop) == [3, 1, 1, 0] and sum(vrt) == 19
    assert ham.eps[:5].max() < ham.eps[5:].min()
    h = ccsd.run_ccsd(ham, cc_conv=10, maxcyc=60, exporder=5)
    assert h["converged"]
    assert -0.22 < h["e_final"] < -0.19


# out.zmat.026 (H2O/DZP, CCSD first-order properties, PROPS=1): the dipole of
# the SCF density (:762-763) and of the correlated density after the
# orbital-relaxation ("iterative expansion of D(ai)", :745) step (:794-795),
# z along the C2 axis, atomic units
GOLD_026_DIPOLE_SCF = 0.8647256373
GOLD_026_DIPOLE_CCSD = 0.8197061290
# electronic second moments <sum r_a r_a> (XX, YY, ZZ) of the same densities
# (:764-765, :796-797); the reference's molecular plane is yz, the fixture's
# xz, so its XX is the fixture's y^2 and its YY the fixture's x^2
GOLD_026_SECOND_SCF = {"x": 7.1867815660, "y": 5.4134779614, "z": 6.4335007706}
GOLD_026_SECOND_CCSD = {"x": 7.3082722125, "y": 5.4731788028, "z": 6.5237129470}


def test_dipoles_match_reference_026():
    """The fixture's MO dipole integrals and SCF orbitals give the reference's
    SCF dipole, and the central finite difference of the oracle's total
    CCSD energy in a field along z, with the SCF re-solved at each field
    (orbital-relaxed), gives the reference's correlated dipole: the relaxed
    CCSD density's dipole is -dE/dF.  Five-point difference at F = +-1e-3,
    +-2e-3 a.u., CCSD to max|dT| < 1e-11."""
    from oracle.hamiltonian import five_point_derivative, scf_in_field
    ham = from_fixture(os.path.join(GOLDEN, "h2o_dzp_zmat026.npz"))
    o = ham.nocc
    mu_scf = ham.nucdip[2] - 2.0 * np.trace(ham.dipole[2][:o, :o])
    assert abs(mu_scf - GOLD_026_DIPOLE_SCF) < 1e-8, mu_scf
    # the field-free SCF of the finite-field code is the fixture's
    e0, h0 = scf_in_field(ham, 0.0)
    assert abs(e0 - ham.e_scf) < 1e-11
    np.testing.assert_allclose(h0.eps, ham.eps, atol=1e-10)

    def e_total(field):
        e_scf, hf = scf_in_field(ham, field)
        return e_scf + ccsd.run_ccsd(hf, cc_conv=11, maxcyc=100, exporder=5)["e_final"]

    mu_ccsd = ham.nucdip[2] - five_point_derivative(e_total, 1e-3)
    assert abs(mu_ccsd - GOLD_026_DIPOLE_CCSD) < 3e-8, mu_ccsd - GOLD_026_DIPOLE_CCSD


def test_zvector_relaxed_density_matches_reference_026():
    """The orbital-relaxed density by the Z-vector method (oracle.relaxed:
    the CC Lagrangian's orbital gradient X(a,i), the RHF response of the
    Brillouin condition, Z^T A = -X; dens/vdens.F:1036-1137) gives the
    reference's correlated dipole and second moments analytically, and the
    dipole's terms add up to the finite-field derivatives of the test above:
    the fixed-orbital CC term Tr(D z) and the orbital-relaxation term
    sum Z_ai z_ai."""
    from oracle.hamiltonian import MOHamiltonian, five_point_derivative
    from oracle import relaxed
    ham = from_fixture(os.path.join(GOLDEN, "h2o_dzp_zmat026.npz"))
    z = ham.dipole[2]
    dens = relaxed.relaxed_density(ham, cc_conv=11)
    p = relaxed.property_derivative(ham, dens, z)
    mu = ham.nucdip[2] - p["total"]
    assert abs(mu - GOLD_026_DIPOLE_CCSD) < 3e-8, mu - GOLD_026_DIPOLE_CCSD
    assert abs(ham.nucdip[2] - p["scf"] - GOLD_026_DIPOLE_SCF) < 1e-8
    # the fixed-orbital CC term against the finite difference of the energy
    # with f -> f + x z (non-HF Fock, orbitals unchanged)
    o = ham.nocc

    def e_fixed(x):
        h = MOHamiltonian(o, ham.fock + x * z, irrep=ham.irrep, eri=ham._eri,
                          nirrep=ham.nirrep)
        return ccsd.run_ccsd(h, cc_conv=12, maxcyc=200, exporder=8)["e_final"]

    assert abs(p["cc"] - five_point_derivative(e_fixed, 1e-3)) < 1e-10
    # the orbital relaxation moves the dipole by 2.53e-3 a.u. here
    assert abs(p["relax"] + 2.5299e-3) < 1e-6
    # the second moments of the SCF and of the relaxed correlated density
    # (the relaxation term is about 1e-2 bohr^2 of each)
    for d, axis in enumerate("xyz"):
        q = relaxed.property_derivative(ham, dens, ham.second[d])
        assert abs(q["scf"] - GOLD_026_SECOND_SCF[axis]) < 1e-8, axis
        assert abs(q["total"] - GOLD_026_SECOND_CCSD[axis]) < 5e-8, (axis, q)
        assert abs(q["relax"]) > 5e-3
