"""GPU test of the largest benchmark system: split-precision CCSD(T) against
the FP64 GPU path at o = 30, v = 270, naux = 900 (the C3 shape, convergent
variant: DF factors scaled by 1/4, seed 2).

This is where the split contractions run their longest sums: the K = v^2 =
72900 products (the T1-dressed <am|ef> tau and <mn|ef> tau terms) take the
256-element FP32 accumulation chunks, and <ab|cd> (42.5 GB of FP64, built on
the device by aces_intprc_df) feeds the packed ladder every cycle.  The
accuracy target of the split path: |dE| <= 1e-6 Eh for the CCSD energy and
for (T).
"""
import pytest

import acesb200 as ab

pytestmark = pytest.mark.gpu


def test_c3_split_ccsd_t_within_1e6_of_fp64():
    import torch
    from acesb200.workloads import WORKLOADS, synthetic_df
    wl = WORKLOADS["c3conv"]
    eps, B, _ = synthetic_df(**wl)
    o, v = wl["nocc"], wl["nvir"]
    lib = ab.load()
    lib.init(0)
    lib.sym_init([o], [v])
    lib.putrec("SCFEVALA", eps)
    dB = torch.from_numpy(B).cuda()
    lib.intprc_df(dB)
    del dB
    torch.cuda.empty_cache()
    exact = lib.xvcc(cc_conv=8, cc_maxcyc=80, cc_exporder=5, triples=1,
                     precision=ab.PREC_FP64)
    split = lib.xvcc(cc_conv=8, cc_maxcyc=80, cc_exporder=5, triples=1,
                     precision=ab.PREC_BF16X3)
    lib.fin()
    assert exact.converged == 1 and split.converged == 1
    d_ccsd = abs(split.e_ccsd - exact.e_ccsd)
    d_t = abs(split.e_t4 + split.e_st5 - exact.e_t4 - exact.e_st5)
    print(f"C3: E(CCSD) {exact.e_ccsd:.10f}, |dE| {d_ccsd:.2e}; E(T) "
          f"{exact.e_t4 + exact.e_st5:.10f}, |dE(T)| {d_t:.2e}; (T) {split.seconds_triples:.3f} s "
          f"split vs {exact.seconds_triples:.3f} s FP64")
    assert d_ccsd <= 1e-6
    assert d_t <= 1e-6
