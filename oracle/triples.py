"""Closed-shell (T) triples correction, restated from the reference's trp/ --
oracle.

Test infrastructure.  The reference's RHF path (trp/trps.F:212,669 ->
trp/trps2.F:242-649) loops over irreps and occupied triplets (i,j,k),
builds the connected triples W_ijk^abc from T2 and the <ab|ci>, <ij|ka>
lists (trp/d1t2new.F:116-584), divides by D_ijk^abc (librt3/rmd314.f,
denominators from librt3/mkd32.F) and accumulates
  E[4]T  = sum (D_ijk - D_abc) t3^2       (trp/e4tijk.F:16-24)
  E[5]ST = the singles term of T1 x t3    (trp/t1t32n.f)
which ``trp/ccenrg.f`` prints; CCSD(T) = CCSD + E[4]T + E[5]ST.

For a closed shell these sums reduce to the spin-free form
  E = 1/3 sum_{ijk,abc} (4 W_abc + W_bca + W_cab)(X_abc - X_cba) / D_ijk^abc
with X = W for E[4]T and X = V - W (the T1-disconnected part
V - W = t_i^a <jk|bc> + t_j^b <ik|ac> + t_k^c <ij|ab>) for E[5]ST.
"""
from __future__ import annotations

import numpy as np


def _connected(t2, g_vvvo, g_ooov, i, j, k):
    """X_ijk^abc = sum_d t(ij,ad) (bd|ck) - sum_l t(il,ab) (ck|jl)."""
    x = np.einsum("ad,bdc->abc", t2[i, j], g_vvvo[:, :, :, k], optimize=True)
    x -= np.einsum("lab,lc->abc", t2[i], g_ooov[:, j, k, :], optimize=True)
    return x


class _Terms:
    """The integral blocks and denominators of one (T) evaluation."""

    def __init__(self, ham, t1, t2, eo=None, ev=None):
        o, v = t1.shape
        self.t1, self.t2 = t1, t2
        self.g_vvvo = ham.chem("vvvo")   # (bd|ck) as [b,d,c,k]
        self.g_ooov = ham.chem("ooov")   # (lj|kc) = (ck|jl) as [l,j,k,c]
        self.g_ovov = ham.chem("ovov")   # (ia|jb) as [i,a,j,b]
        if eo is None:
            eps = ham.eps
            eo, ev = eps[:o], eps[o:]
        self.eo = eo
        self.Dabc = ev[:, None, None] + ev[None, :, None] + ev[None, None, :]

    def ordered(self, i, j, k):
        """3 x the contribution of the ordered triplet (i, j, k) to (E[4]T, E[5]ST)."""
        t1, t2, gv, go, gd = self.t1, self.t2, self.g_vvvo, self.g_ooov, self.g_ovov
        W = (_connected(t2, gv, go, i, j, k)
             + _connected(t2, gv, go, i, k, j).transpose(0, 2, 1)
             + _connected(t2, gv, go, j, i, k).transpose(1, 0, 2)
             + _connected(t2, gv, go, j, k, i).transpose(2, 0, 1)
             + _connected(t2, gv, go, k, i, j).transpose(1, 2, 0)
             + _connected(t2, gv, go, k, j, i).transpose(2, 1, 0))
        Vd = (np.einsum("a,bc->abc", t1[i], gd[j, :, k, :])
              + np.einsum("b,ac->abc", t1[j], gd[i, :, k, :])
              + np.einsum("c,ab->abc", t1[k], gd[i, :, j, :]))
        D = self.eo[i] + self.eo[j] + self.eo[k] - self.Dabc
        Z = (4.0 * W + W.transpose(2, 0, 1) + W.transpose(1, 2, 0)) / D
        return np.sum(Z * (W - W.transpose(2, 1, 0))), np.sum(Z * (Vd - Vd.transpose(2, 1, 0)))


def triples(ham, t1, t2, eo=None, ev=None, return_parts=False):
    """Returns (E[4]T, E[5]ST) for converged closed-shell CCSD amplitudes."""
    o = t1.shape[0]
    T = _Terms(ham, t1, t2, eo, ev)
    e4 = 0.0
    e5 = 0.0
    for i in range(o):
        for j in range(o):
            for k in range(o):
                a4, a5 = T.ordered(i, j, k)
                e4 += a4
                e5 += a5
    return e4 / 3.0, e5 / 3.0


def triples_unique(ham, t1, t2, triplets, eo=None, ev=None):
    """(E[4]T, E[5]ST) restricted to the given triplets i >= j >= k, each
    standing for its distinct orderings (the unit the engine distributes over
    GPUs): summed over all triplets this equals `triples`."""
    import itertools
    T = _Terms(ham, t1, t2, eo, ev)
    e4 = 0.0
    e5 = 0.0
    for (i, j, k) in triplets:
        for p in set(itertools.permutations((i, j, k))):
            a4, a5 = T.ordered(*p)
            e4 += a4
            e5 += a5
    return e4 / 3.0, e5 / 3.0
