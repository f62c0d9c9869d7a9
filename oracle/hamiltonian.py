"""Closed-shell MO Hamiltonians for the oracle (test infrastructure).

Two sources:

* ``from_fixture``: the H2O/DZP fixtures in tests/golden (orbital energies and
  MO integrals produced by tests/golden/make_h2o_dzp.py);
* ``synthetic``: the seeded density-fitted generator of the benchmark
  workloads -- occupied energies U[-1.5,-0.3], virtual energies U[0.2,3.0],
  (pq|rs) = sum_L B^L_pq B^L_rs with B symmetric in pq and N(0, 0.02^2)
  entries, Fock = diag(eps).

Integral blocks are returned in physicists' notation v[p,q,r,s] = <pq|rs> =
(pr|qs), the convention of the reference's MOINTS lists (intprc/clmoio.F).
"""
from __future__ import annotations

import numpy as np


class MOHamiltonian:
    """Orbital energies / Fock matrix plus chemists'-notation integral access.

    Orbitals are ordered occupied first, then virtual; within each block by
    irrep (the reference's DPD order).  ``irrep`` holds the 0-based irrep of
    every orbital (all zero for C1).
    """

    def __init__(self, nocc, fock, irrep=None, eri=None, df=None, nirrep=1):
        self.nocc = int(nocc)
        self.fock = np.asarray(fock, dtype=np.float64)
        self.nmo = self.fock.shape[0]
        self.nvir = self.nmo - self.nocc
        self.irrep = np.zeros(self.nmo, dtype=np.int64) if irrep is None else np.asarray(irrep)
        self.nirrep = int(nirrep)
        self._eri = eri      # full (pq|rs) tensor, or None
        self._df = df        # B[L, p, q], or None
        self._cache = {}

    # ---- orbital data ---------------------------------------------------
    @property
    def eps(self):
        return np.diag(self.fock).copy()

    def pop_vrt(self):
        o = self.nocc
        pop = np.array([np.sum(self.irrep[:o] == h) for h in range(self.nirrep)])
        vrt = np.array([np.sum(self.irrep[o:] == h) for h in range(self.nirrep)])
        return pop, vrt

    # ---- integrals --------------------------------------------------------
    def _sl(self, c):
        o = self.nocc
        return slice(0, o) if c == "o" else slice(o, self.nmo)

    def chem(self, key):
        """(pq|rs) block, key like 'ovov' (chemists' notation)."""
        if key in self._cache:
            return self._cache[key]
        s = [self._sl(c) for c in key]
        if self._eri is not None:
            out = np.ascontiguousarray(self._eri[s[0], s[1], s[2], s[3]])
        else:
            B = self._df
            L1 = B[:, s[0], s[1]].reshape(B.shape[0], -1)
            L2 = B[:, s[2], s[3]].reshape(B.shape[0], -1)
            out = (L1.T @ L2).reshape(B[:, s[0], s[1]].shape[1:] + B[:, s[2], s[3]].shape[1:])
        self._cache[key] = out
        return out

    def phys(self, key):
        """<pq|rs> block, key like 'oovv' -> v[p,q,r,s] = (pr|qs)."""
        k = "phys" + key
        if k in self._cache:
            return self._cache[k]
        c = self.chem(key[0] + key[2] + key[1] + key[3])
        out = np.ascontiguousarray(c.transpose(0, 2, 1, 3))
        self._cache[k] = out
        return out

    def drop_cache(self):
        self._cache = {}


def unpack8(e8, n):
    """Inverse of the fixture's 8-fold packing of (pq|rs)."""
    tri = [(p, q) for p in range(n) for q in range(p + 1)]
    npair = len(tri)
    M = np.zeros((npair, npair))
    iu = np.tril_indices(npair)
    M[iu] = e8
    M = M + M.T - np.diag(np.diag(M))
    idx = np.array(tri)
    pair_of = np.zeros((n, n), dtype=np.int64)
    pair_of[idx[:, 0], idx[:, 1]] = np.arange(npair)
    pair_of[idx[:, 1], idx[:, 0]] = np.arange(npair)
    return M[pair_of[:, :, None, None], pair_of[None, None, :, :]]


def from_fixture(path):
    d = np.load(path)
    n = int(d["nmo"])
    g = unpack8(d["eri8"], n)
    pop = d["pop"]
    nocc = int(pop.sum())
    ham = MOHamiltonian(nocc, np.diag(d["eps"]), irrep=d["irrep"], eri=g, nirrep=len(pop))
    ham.e_scf = float(d["e_scf"])
    ham.e_nuc = float(d["e_nuc"])
    ham.dipole = d["dipole"]
    ham.nucdip = d["nucdip"]
    return ham


def synthetic_factors(nocc, nvir, naux, seed, irreps=None, bscale=1.0):
    """Seeded DF factors of the synthetic workloads: the generator of the
    engine's benchmark package (acesb200.workloads.synthetic_df), so the oracle
    and the engine see bit-identical inputs."""
    import os
    import sys
    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "aces-ii_b200")
    if pkg not in sys.path:
        sys.path.insert(0, pkg)
    from acesb200.workloads import synthetic_df
    return synthetic_df(nocc, nvir, naux, seed, irreps, bscale)


def synthetic(nocc, nvir, naux, seed, irreps=None, bscale=1.0):
    eps, B, irr = synthetic_factors(nocc, nvir, naux, seed, irreps, bscale)
    return MOHamiltonian(nocc, np.diag(eps), irrep=irr, df=B, nirrep=irreps or 1)
