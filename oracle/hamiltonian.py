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
    ham.hcore = d["hcore"]
    if "second" in d.files:   # diagonal second moments x^2, y^2, z^2 (MO basis)
        ham.second = d["second"]
        ham.nucsecond = d["nucsecond"]
    return ham


def scf_in_field(ham, field, axis=2, tol=1e-12, maxit=200):
    """RHF of a fixture molecule in a uniform electric field along ``axis``
    (test infrastructure for finite-field dipoles).

    The one-electron operator becomes h + field * r_axis (r the electronic
    position; the field's interaction with the nuclei, -field * sum_A Z_A
    R_A,axis, is a constant left out, so the dipole is nucdip - dE/dfield).
    Works in the basis of the zero-field MOs, which is orthonormal and spans
    the AO space, from the fixture's core Hamiltonian, MO integrals and MO
    dipole integrals; Roothaan steps with DIIS (8 vectors), each irrep's
    block diagonalised on its own so the orbitals keep their irreps (a field
    along the C2 axis of a C2v molecule is totally symmetric), the lowest
    pop[h] orbitals of irrep h occupied.  The reference's SCF program
    (vscf/) is out of scope of the engine; this restates plain RHF only to
    make the field-dependent orbitals of a finite-difference check.

    Returns (E_SCF electronic + nuclear repulsion, MOHamiltonian in the
    field's canonical orbitals, DPD order: occupied by irrep, then virtual by
    irrep, energy order within)."""
    n, o = ham.nmo, ham.nocc
    g = ham._eri
    hF = ham.hcore + field * ham.dipole[axis]
    irr = np.asarray(ham.irrep)
    pop, _ = ham.pop_vrt()
    blocks = [np.where(irr == h)[0] for h in range(ham.nirrep)]

    def canonical(F):
        eps = np.zeros(n)
        C = np.zeros((n, n))
        for idx in blocks:
            w, v = np.linalg.eigh(F[np.ix_(idx, idx)])
            C[np.ix_(idx, idx)] = v
            eps[idx] = w
        occ = [i for h, idx in enumerate(blocks) for i in idx[:pop[h]]]
        vir = [i for h, idx in enumerate(blocks) for i in idx[pop[h]:]]
        order = occ + vir
        return eps[order], C[:, order]

    Cocc = np.eye(n)[:, :o]
    focks, errs = [], []
    for _ in range(maxit):
        D = 2.0 * Cocc @ Cocc.T
        F = hF + np.einsum("pqrs,rs->pq", g, D) - 0.5 * np.einsum("prqs,rs->pq", g, D)
        err = F @ D - D @ F
        if np.abs(err).max() < tol:
            break
        focks.append(F)
        errs.append(err)
        focks, errs = focks[-8:], errs[-8:]
        m = len(focks)
        Bm = -np.ones((m + 1, m + 1))
        Bm[m, m] = 0.0
        for i in range(m):
            for j in range(m):
                Bm[i, j] = np.sum(errs[i] * errs[j])
        rhs = np.zeros(m + 1)
        rhs[m] = -1.0
        c = np.linalg.solve(Bm, rhs)
        _, C = canonical(sum(c[i] * focks[i] for i in range(m)))
        Cocc = C[:, :o]
    else:
        raise RuntimeError("scf_in_field: no convergence")
    e_scf = 0.5 * np.sum(D * (hF + F)) + ham.e_nuc
    eps, C = canonical(F)
    eri = np.einsum("pqrs,pi,qj,rk,sl->ijkl", g, C, C, C, C, optimize=True)
    out = MOHamiltonian(o, np.diag(eps), irrep=irr[np.argmax(np.abs(C), axis=0)], eri=eri,
                        nirrep=ham.nirrep)
    out.e_scf = e_scf
    return e_scf, out


def five_point_derivative(f, delta):
    """df/dx at 0 from f(+-delta), f(+-2 delta) (error O(delta^4))."""
    return (8.0 * (f(delta) - f(-delta)) - (f(2 * delta) - f(-2 * delta))) / (12.0 * delta)


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
