"""GPU tests of the device MO-integral list producer (aces_intprc_df), the
B200 counterpart of the reference's vtran + intprc chain for density-fitted
or Cholesky-decomposed MO integrals (intprc/clmoio.F:46-260).

* C1 and 8-irrep synthetic systems: every irrep block of lists 13, 10, 16,
  25, 30 and 233 equals the list the oracle's dense integrals give through
  PUTLST (same layout, values to FP64 rounding of the L sum);
* H2O/DZP (C2v): the reference-geometry integrals factorised by an exact
  pivoted Cholesky decomposition on the host give, through the producer,
  the golden CCSD energy of out.zmat.035.ccsd:628.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
import acesb200 as ab
from acesb200 import INTEGRAL_LISTS
from oracle.hamiltonian import from_fixture, synthetic, synthetic_factors
from oracle import ccsd
from test_gpu_ccsd import setup_lists

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    lib = ab.load()
    lib.init(0)
    return lib


def snapshot(lib):
    out = {}
    for lst in INTEGRAL_LISTS:
        for h in range(1, lib.nirrep + 1):
            nr, nc = lib.list_dims(h, lst)
            out[(lst, h)] = lib.getlst(1, nc, h, lst) if nr * nc else np.zeros((nr, nc))
    return out


def lists_from_producer(lib, eps, B, irr, o):
    lib.init(0)
    pop = [int(np.sum(irr[:o] == h)) for h in range(max(irr) + 1)]
    vrt = [int(np.sum(irr[o:] == h)) for h in range(max(irr) + 1)]
    lib.sym_init(pop, vrt)
    lib.putrec("SCFEVALA", np.asarray(eps, dtype=np.float64))
    lib.intprc_df(np.ascontiguousarray(B))


@pytest.mark.parametrize("o,v,naux,seed,irreps", [(6, 24, 40, 5, None), (7, 33, 56, 1006, 8)])
def test_producer_lists_equal_putlst_lists(lib, o, v, naux, seed, irreps):
    eps, B, irr = synthetic_factors(o, v, naux, seed, irreps)
    ham = synthetic(o, v, naux, seed, irreps=irreps)
    setup_lists(lib, ham)
    ref = snapshot(lib)
    lists_from_producer(lib, eps, B, irr, o)
    got = snapshot(lib)
    assert got.keys() == ref.keys()
    scale = max(np.abs(x).max() for x in ref.values() if x.size)
    for key in ref:
        assert got[key].shape == ref[key].shape, key
        if ref[key].size:
            assert np.abs(got[key] - ref[key]).max() <= 1e-14 * scale, key
    cfg = lib.xvcc(cc_conv=10, cc_maxcyc=80, cc_exporder=5)
    e = ccsd.run_ccsd(ham, cc_conv=10, maxcyc=80, exporder=5)["e_final"]
    assert abs(cfg.e_ccsd - e) < 1e-11


def cholesky_factors(g, tol=1e-13):
    """Pivoted Cholesky of the (pq|rs) supermatrix: B[L, p, q] with
    sum_L B[L,p,q] B[L,r,s] = (pq|rs) to tol."""
    n = g.shape[0]
    M = g.reshape(n * n, n * n)
    d = np.diag(M).copy()
    vecs = []
    while True:
        k = int(np.argmax(d))
        if d[k] < tol:
            break
        col = M[:, k].copy()
        for L in vecs:
            col -= L * L[k]
        L = col / np.sqrt(d[k])
        vecs.append(L)
        d -= L * L
    return np.array(vecs).reshape(len(vecs), n, n)


def test_producer_on_cholesky_factors_reaches_the_golden_energy(lib):
    ham = from_fixture(os.path.join(GOLDEN, "h2o_dzp_zmat035.npz"))
    g = ham._eri
    B = cholesky_factors(g)
    B = 0.5 * (B + B.transpose(0, 2, 1))
    assert np.abs(np.einsum("Lpq,Lrs->pqrs", B, B) - g).max() < 1e-12
    lists_from_producer(lib, ham.eps, B, np.asarray(ham.irrep), ham.nocc)
    cfg = lib.xvcc(cc_conv=7, cc_maxcyc=50, cc_exporder=5)
    assert cfg.ncycle == 11
    assert abs(cfg.e_ccsd - (-0.226005606663)) < 1e-10


def test_producer_from_a_device_tensor_and_errors(lib):
    import torch
    o, v, naux, seed = 5, 20, 30, 9
    eps, B, irr = synthetic_factors(o, v, naux, seed)
    lib.init(0)
    lib.sym_init([o], [v])
    lib.putrec("SCFEVALA", eps)
    lib.intprc_df(torch.from_numpy(B).cuda())
    dev = snapshot(lib)
    lists_from_producer(lib, eps, B, irr, o)
    host = snapshot(lib)
    for key in host:
        np.testing.assert_array_equal(dev[key], host[key])
    lib.init(0)
    with pytest.raises(ab.AcesError) as e:     # no symmetry yet
        lib.intprc_df(B)
    assert e.value.status == -7
