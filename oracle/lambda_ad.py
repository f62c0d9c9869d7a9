"""Lambda equations and the CCSD one-particle density by automatic
differentiation -- oracle (test infrastructure).

The reference solves the Lambda (left-hand) CC equations in xlambda
(lambda/vlamcc.F:597-927, terms listed in lambda/README) and forms the
one-particle density in xdens (dens/densoo.F, densvv.F, densvo.F).  Both are
derivatives of the CC Lagrangian

    L(T, lambda, f) = E(T, f) + lambda . r(T, f),    r = Z(T) - D(f) o T,

with Z the increments of oracle.ccsd.residual and D the orbital-energy
denominators.  This module evaluates the same residual with torch tensors and
lets torch autograd supply the derivatives, independently of the engine's
hand-written backward kernels:

  * lambda solves (dr/dT)^T lambda = -dE/dT exactly (full Jacobian; small
    systems only);
  * D_pq = dL/df_pq at fixed orbitals and integrals, so that for a
    perturbation f -> f + x h' the energy derivative is dE/dx = Tr(D h').
"""
from __future__ import annotations

import numpy as np

from . import ccsd


class TorchBlocks:
    """Blocks of oracle.ccsd with torch tensors; the Fock blocks are leaves."""

    def __init__(self, B, torch):
        self.o, self.v = B.o, B.v
        T = lambda x: torch.tensor(np.ascontiguousarray(x), dtype=torch.float64)
        for k in ("oooo", "ooov", "oovv", "ovvo", "ovov", "ovvv", "vvvv"):
            setattr(self, k, T(getattr(B, k)))
        self.foo = T(B.foo).requires_grad_(True)
        self.fvv = T(B.fvv).requires_grad_(True)
        self.fov = T(B.fov).requires_grad_(True)
        self.refresh()

    def refresh(self):
        import torch
        self.eo = torch.diagonal(self.foo)
        self.ev = torch.diagonal(self.fvv)
        self.Dov = self.eo[:, None] - self.ev[None, :]
        self.Doovv = (self.eo[:, None, None, None] + self.eo[None, :, None, None]
                      - self.ev[None, None, :, None] - self.ev[None, None, None, :])


def _energy(TB, t1, t2):
    import torch
    tau = t2 + torch.einsum("ia,jb->ijab", t1, t1)
    L = 2.0 * TB.oovv - TB.oovv.permute(0, 1, 3, 2)
    return torch.sum(L * tau) + 2.0 * torch.sum(TB.fov * t1)


def _r(TB, t1, t2):
    Z1, Z2 = ccsd.residual(TB, t1, t2)
    return Z1 - TB.Dov * t1, Z2 - TB.Doovv * t2


def solve_lambda(B, t1, t2, symmetric=True):
    """Returns (l1, l2) solving (dr/dT)^T lambda = -dE/dT.

    With ``symmetric`` (the reference's and the engine's convention: T2 and
    lambda2 carry the pair symmetry t(ij,ab) = t(ji,ba), enforced after every
    update by SYMETRIZE_T2, vcc/dodiis0.F:57) the equations are solved in that
    subspace: P J^T P lambda = -P g with P the symmetriser."""
    import torch
    TB = TorchBlocks(B, torch)
    o, v = B.o, B.v
    n1, n2 = o * v, o * o * v * v
    t1t = torch.tensor(t1, dtype=torch.float64)
    t2t = torch.tensor(t2, dtype=torch.float64)

    def rvec(x):
        a, b = _r(TB, x[:n1].reshape(o, v), x[n1:].reshape(o, o, v, v))
        return torch.cat([a.reshape(-1), b.reshape(-1)])

    x0 = torch.cat([t1t.reshape(-1), t2t.reshape(-1)]).detach()
    J = torch.autograd.functional.jacobian(rvec, x0, vectorize=True)
    xg = x0.clone().requires_grad_(True)
    e = _energy(TB, xg[:n1].reshape(o, v), xg[n1:].reshape(o, o, v, v))
    (g,) = torch.autograd.grad(e, xg)
    if symmetric:
        n = n1 + n2
        idx = torch.arange(n2).reshape(o, o, v, v).permute(1, 0, 3, 2).reshape(-1)
        P = torch.zeros(n, n, dtype=torch.float64)
        P[:n1, :n1] = torch.eye(n1, dtype=torch.float64)
        P[n1 + torch.arange(n2), n1 + torch.arange(n2)] += 0.5
        P[n1 + torch.arange(n2), n1 + idx] += 0.5
        M = P @ J.T @ P + (torch.eye(n, dtype=torch.float64) - P)
        lam = torch.linalg.solve(M, -(P @ g))
    else:
        lam = torch.linalg.solve(J.T, -g)
    lam = lam.detach().numpy()
    return lam[:n1].reshape(o, v), lam[n1:].reshape(o, o, v, v)


def density(B, t1, t2, l1, l2):
    """D_pq = dL/df_pq (occupied-occupied, virtual-virtual, occupied-virtual
    blocks; the engine reads f_ov only, so D_vo = 0)."""
    import torch
    TB = TorchBlocks(B, torch)
    t1t = torch.tensor(t1, dtype=torch.float64)
    t2t = torch.tensor(t2, dtype=torch.float64)
    l1t = torch.tensor(l1, dtype=torch.float64)
    l2t = torch.tensor(l2, dtype=torch.float64)
    r1, r2 = _r(TB, t1t, t2t)
    Lag = _energy(TB, t1t, t2t) + torch.sum(l1t * r1) + torch.sum(l2t * r2)
    goo, gvv, gov = torch.autograd.grad(Lag, [TB.foo, TB.fvv, TB.fov])
    o, v = B.o, B.v
    D = np.zeros((o + v, o + v))
    D[:o, :o] = goo.numpy()
    D[o:, o:] = gvv.numpy()
    D[:o, o:] = gov.numpy()
    return D
