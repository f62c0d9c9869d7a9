"""Seeded synthetic closed-shell MO Hamiltonians (the benchmark workloads).

Generator of the synthetic systems: occupied orbital energies U[-1.5,-0.3],
virtual U[0.2,3.0] (Eh), density-fitted two-electron integrals
(pq|rs) = sum_L B^L_pq B^L_rs with B symmetric in pq and N(0, 0.02^2) entries,
Fock = diag(eps).  With ``irreps`` > 1 orbitals are dealt into irreps
unevenly, every auxiliary function carries an irrep and B^L_pq = 0 unless
irrep(p) ^ irrep(q) == irrep(L), which keeps (pq|rs) symmetry-consistent;
orbitals are then ordered by irrep (energy order inside an irrep), the
reference's DPD orbital order.

Named workloads (nocc, nvir, naux, seed):
  * ``c1`` ... (H2O/cc-pVDZ shape) is not synthetic; see tests/golden.
  * ``c2``: 20, 180, 600, seed 1 -- the CCSD s/iter benchmark system;
  * ``c3``: 30, 270, 900, seed 2 -- CCSD(T);
  * ``c4``: 20, 180, 600, seed 3 -- Lambda + density;
  * ``c5``: 64 systems, nocc 4-24, nvir 30-220, 8 irreps, seeds 1000+k.
"""
from __future__ import annotations

import numpy as np

WORKLOADS = {
    "c2": dict(nocc=20, nvir=180, naux=600, seed=1),
    "c3": dict(nocc=30, nvir=270, naux=900, seed=2),
    "c4": dict(nocc=20, nvir=180, naux=600, seed=3),
    # The systems above, taken literally, have CC equations whose Jacobi/DIIS
    # iteration diverges (the <ab|cd> coupling naux*sigma^2*nvir ~ 20 Eh exceeds
    # the ~5 Eh denominators).  The "conv" variants scale B by 1/4 (entries
    # N(0, 0.005^2)), same shapes, and converge; they carry the accuracy figures.
    "c2conv": dict(nocc=20, nvir=180, naux=600, seed=1, bscale=0.25),
    "c3conv": dict(nocc=30, nvir=270, naux=900, seed=2, bscale=0.25),
    "c4conv": dict(nocc=20, nvir=180, naux=600, seed=3, bscale=0.25),
}


def synthetic_df(nocc, nvir, naux, seed, irreps=None, bscale=1.0):
    """Returns (eps[nmo], B[naux, nmo, nmo], orbital irreps[nmo])."""
    rng = np.random.default_rng(seed)
    eo = np.sort(rng.uniform(-1.5, -0.3, nocc))
    ev = np.sort(rng.uniform(0.2, 3.0, nvir))
    nmo = nocc + nvir
    B = rng.normal(0.0, 0.02, (naux, nmo, nmo))
    B = 0.5 * (B + B.transpose(0, 2, 1))
    if bscale != 1.0:
        B *= bscale
    eps = np.concatenate([eo, ev])
    if irreps and irreps > 1:
        w = rng.uniform(0.5, 1.5, irreps)
        w = w / w.sum()
        occ_irr = rng.choice(irreps, nocc, p=w)
        vir_irr = rng.choice(irreps, nvir, p=w)
        orb_irr = np.concatenate([occ_irr, vir_irr])
        aux_irr = rng.integers(0, irreps, naux)
        mask = (orb_irr[:, None] ^ orb_irr[None, :])[None, :, :] == aux_irr[:, None, None]
        B = B * mask
        order_o = np.lexsort((eps[:nocc], occ_irr))
        order_v = nocc + np.lexsort((eps[nocc:], vir_irr))
        order = np.concatenate([order_o, order_v])
        eps = eps[order]
        orb_irr = orb_irr[order]
        B = B[:, order][:, :, order]
    else:
        orb_irr = np.zeros(nmo, dtype=np.int64)
    return eps, B, orb_irr


def batch_systems(nsys=64, base_seed=1000):
    """The 64-system batch: nocc ~ U{4..24}, nvir ~ U{30..220}, 8 irreps."""
    rng = np.random.default_rng(base_seed)
    out = []
    for k in range(nsys):
        o = int(rng.integers(4, 25))
        v = int(rng.integers(30, 221))
        out.append(dict(nocc=o, nvir=v, naux=max(2 * (o + v), 64), seed=base_seed + k, irreps=8))
    return out
