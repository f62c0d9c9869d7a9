"""CPU test: the EOM-CCSD oracle pinned to the reference's golden excitation
energies.

test/OUTPUT/out.zmat.035.ccsd (H2O/DZP, R = 0.957 A, A = 104.5 deg,
EXCITE=EOMEE, ESTATE_SYM=1/1/1/1) prints one singlet EOM-CCSD root per C2v
irrep as total EOM-CCSD energies (:860, :972, :1090, :1202); with the CCSD
total energy of the same run (TEST.DAT TOTENERG -76.2725089278) they give the
excitation energies below.  The reference converges its Davidson roots to
about 1e-7 Eh (its two passes over irrep 1 differ by 4e-8 Eh), hence 1e-7.
"""
import os

import pytest

from conftest import GOLDEN
from oracle.hamiltonian import from_fixture
from oracle import ccsd, eom

E_CCSD_TOTAL = -76.2725089278
GOLD_EOM_TOTAL = [-75.843373150515, -75.939268816118, -75.756716770718, -75.863723085307]
GOLD_OMEGA = [e - E_CCSD_TOTAL for e in GOLD_EOM_TOTAL]


def test_eom_ccsd_h2o_dzp_matches_reference():
    ham = from_fixture(os.path.join(GOLDEN, "h2o_dzp_zmat035.npz"))
    h = ccsd.run_ccsd(ham, cc_conv=10, maxcyc=60, exporder=5)
    assert abs(ham.e_scf + h["e_final"] - E_CCSD_TOTAL) < 5e-9   # the reference stopped at 1e-7
    w = eom.eom_ccsd(ham, h["t1"], h["t2"], [1, 1, 1, 1], tol=1e-7)
    for irrep in range(4):
        assert abs(w[irrep][0] - GOLD_OMEGA[irrep]) < 1e-7, (irrep, w[irrep][0])
    # 11.6774, 9.0679, 14.0354, 11.1236 eV as printed (:885, :998, :1117, :1227)
    ev = [27.2113957 * w[h_][0] for h_ in range(4)]
    assert [round(x, 4) for x in ev] == [11.6774, 9.0679, 14.0354, 11.1236]
