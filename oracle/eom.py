"""EOM-EE-CCSD singlet excitation energies -- oracle (test infrastructure).

The reference computes them in xvee: for each irrep (vee/doeomee_david.F:99-
300) it forms the diagonal of the similarity-transformed Hamiltonian
(HBARDIAG), a Tamm-Dancoff guess (NEWGES), and runs a Davidson iteration
whose products are Hbar times the trial vectors (HBARXC) with NEXTDAV
extrapolating the subspace; right- and left-hand eigenvectors give the same
eigenvalues.

Restated here: in the closed-shell spin-adapted parametrisation of
oracle.ccsd (t1[i,a], t2[i,j,a,b] = t_iJ^aB with the pair symmetry
t2[i,j,a,b] = t2[j,i,b,a]) the residual is r(T) = Z(T) - D o T, and its
Jacobian J = dr/dT restricted to the pair-symmetric subspace is the singlet
block of Hbar - E_CC over the single and double excitations: its eigenvalues
are the singlet EOM-CCSD excitation energies.  This module runs a Davidson
iteration on the TRANSPOSED Jacobian P J^T P (P: the pair symmetriser, an
orthogonal projector, so P J^T P is the transpose of P J P on that subspace
and shares its eigenvalues), with the products J^T x from torch autograd --
independently of the engine's hand-written backward kernels.  A state of
irrep h has amplitudes only on the excitations whose orbital irreps multiply
to h.
"""
from __future__ import annotations

import numpy as np

from . import ccsd
from .lambda_ad import TorchBlocks


def irrep_masks(irr_o, irr_v, h):
    """0/1 masks of the singles [o, v] and doubles [o, o, v, v] of irrep h."""
    io, iv = np.asarray(irr_o), np.asarray(irr_v)
    m1 = ((io[:, None] ^ iv[None, :]) == h).astype(float)
    m2 = ((io[:, None, None, None] ^ io[None, :, None, None]
           ^ iv[None, None, :, None] ^ iv[None, None, None, :]) == h).astype(float)
    return m1, m2


def eom_ccsd(ham, t1, t2, nroots, tol=1e-7, maxit=80, log=None):
    """Lowest ``nroots[h]`` singlet EOM-CCSD excitation energies (Eh) of every
    irrep h at the converged amplitudes (t1, t2).  Returns {h: [omega, ...]}."""
    import torch
    B = ccsd.Blocks(ham)
    TB = TorchBlocks(B, torch)
    o, v = B.o, B.v
    t1t = torch.tensor(t1, dtype=torch.float64, requires_grad=True)
    t2t = torch.tensor(ccsd.symmetrize_t2(np.asarray(t2, dtype=float)), dtype=torch.float64,
                       requires_grad=True)
    Z1, Z2 = ccsd.residual(TB, t1t, t2t)
    D1, D2 = TB.Dov.detach().numpy(), TB.Doovv.detach().numpy()
    n1 = o * v
    irr = np.asarray(ham.irrep)
    irr_o, irr_v = irr[:o], irr[o:]

    def split(x):
        return x[:n1].reshape(o, v), x[n1:].reshape(o, o, v, v)

    def join(a, b):
        return np.concatenate([a.ravel(), b.ravel()])

    def sigma(x):
        a, b = split(x)
        ga, gb = torch.autograd.grad([Z1, Z2], [t1t, t2t], [torch.tensor(a), torch.tensor(b)],
                                     retain_graph=True)
        return join(ga.numpy() - D1 * a, ccsd.symmetrize_t2(gb.numpy()) - D2 * b)

    diag = join(-D1, -D2)
    out = {}
    for h, k in enumerate(nroots):
        if k <= 0:
            continue
        m1, m2 = irrep_masks(irr_o, irr_v, h)
        mask = join(m1, m2)
        # guesses: the singles of this irrep with the smallest orbital-energy gaps
        cand = np.flatnonzero(join(m1, np.zeros_like(m2)))
        cand = cand[np.argsort(diag[cand])][:max(2 * k, k + 2)]
        V = []
        for c in cand:
            e = np.zeros(mask.size)
            e[c] = 1.0
            V.append(e)
        S = [sigma(x) for x in V]
        omega = np.zeros(k)
        conv = False
        for it in range(maxit):
            Vm, Sm = np.array(V), np.array(S)
            G = Vm @ Sm.T                       # G[i, j] = v_i . (A v_j)
            w, Y = np.linalg.eig(G)             # A restricted: (V A V^T) y = w y
            order = np.argsort(w.real)
            w, Y = w[order].real, Y[:, order].real
            new = []
            done = True
            for r in range(k):
                y = Y[:, r]
                x = y @ Vm
                res = y @ Sm - w[r] * x
                if np.linalg.norm(res) > tol or abs(w[r] - omega[r]) > tol:
                    done = False
                    den = w[r] - diag
                    den[np.abs(den) < 1e-2] = 1e-2
                    d = mask * res / den
                    d = join(*(lambda a, b: (a, ccsd.symmetrize_t2(b)))(*split(d)))
                    new.append(d)
            omega = w[:k].copy()
            if log:
                log(f"irrep {h + 1} iter {it + 1} dim {len(V)} omega {omega}")
            if done:
                conv = True
                break
            for d in new:
                for _ in range(2):
                    for q in V:
                        d = d - (q @ d) * q
                nd = np.linalg.norm(d)
                if nd > 1e-10:
                    V.append(d / nd)
                    S.append(sigma(V[-1]))
        if not conv:
            raise RuntimeError(f"EOM Davidson did not converge for irrep {h + 1}")
        out[h] = list(omega)
    return out
