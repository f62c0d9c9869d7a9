"""CPU oracle for the CCSD / (T) / Lambda hot path -- TEST INFRASTRUCTURE ONLY.

This package restates the reference's algorithms (ACES II ``vcc/``, ``libr/``,
``libr2/``, ``trp/``, ``lambda/``, ``dens/``) in FP64 numpy so that the CUDA
engine can be checked against it.  Only ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` may import it, and only as the
checker or as the timed CPU baseline; the engine itself never calls into it.

Parity pins (see tests/test_oracle_golden.py):
  * H2O/DZP SCF, MP2 and every CCSD iteration energy of the reference's
    regression run test/OUTPUT/out.zmat.035.ccsd:443,555-650;
  * H2O/DZP CCSD + (T) energies of test/OUTPUT/out.zmat.020:650-688.
"""
