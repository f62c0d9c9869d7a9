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


def triples(ham, t1, t2, eo=None, ev=None, return_parts=False):
    """Returns (E[4]T, E[5]ST) for converged closed-shell CCSD amplitudes."""
    o, v = t1.shape
    g_vvvo = ham.chem("vvvo")   # (bd|ck) as [b,d,c,k]
    g_ooov = ham.chem("ooov")   # (lj|kc) = (ck|jl) as [l,j,k,c]
    g_ovov = ham.chem("ovov")   # (ia|jb) as [i,a,j,b]
    if eo is None:
        eps = ham.eps
        eo, ev = eps[:o], eps[o:]
    Dabc = ev[:, None, None] + ev[None, :, None] + ev[None, None, :]
    e4 = 0.0
    e5 = 0.0
    for i in range(o):
        for j in range(o):
            for k in range(o):
                W = (_connected(t2, g_vvvo, g_ooov, i, j, k)
                     + _connected(t2, g_vvvo, g_ooov, i, k, j).transpose(0, 2, 1)
                     + _connected(t2, g_vvvo, g_ooov, j, i, k).transpose(1, 0, 2)
                     + _connected(t2, g_vvvo, g_ooov, j, k, i).transpose(2, 0, 1)
                     + _connected(t2, g_vvvo, g_ooov, k, i, j).transpose(1, 2, 0)
                     + _connected(t2, g_vvvo, g_ooov, k, j, i).transpose(2, 1, 0))
                Vd = (np.einsum("a,bc->abc", t1[i], g_ovov[j, :, k, :])
                      + np.einsum("b,ac->abc", t1[j], g_ovov[i, :, k, :])
                      + np.einsum("c,ab->abc", t1[k], g_ovov[i, :, j, :]))
                D = eo[i] + eo[j] + eo[k] - Dabc
                Z = (4.0 * W + W.transpose(2, 0, 1) + W.transpose(1, 2, 0)) / D
                e4 += np.sum(Z * (W - W.transpose(2, 1, 0)))
                e5 += np.sum(Z * (Vd - Vd.transpose(2, 1, 0)))
    return e4 / 3.0, e5 / 3.0
