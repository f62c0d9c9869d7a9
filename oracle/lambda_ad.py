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


def lambda_to_reference(l1, l2):
    """The reference's closed-shell multipliers (lists 190 and 146, the
    alpha-beta block) from this module's: lambda = dL/dr for the spin-adapted
    residual r of oracle.ccsd, l1 = 2 L1 and l2 = 2 L2 - L2~ (L2~: virtuals
    swapped), so L1 = l1 / 2 and L2 = (2 l2 + l2~) / 3."""
    return 0.5 * l1, (2.0 * l2 + l2.transpose(0, 1, 3, 2)) / 3.0


def lambda_from_reference(L1, L2):
    """Inverse of lambda_to_reference."""
    return 2.0 * L1, 2.0 * L2 - L2.transpose(0, 1, 3, 2)


def iterate_lambda(B, t1, t2, cc_conv=7, maxcyc=50, exporder=5):
    """The xlambda cycle (lambda/vlamcc.F:597-927) as the reference runs it:
    multipliers kept in the reference's convention (lambda_to_reference),
    started from the converged amplitudes (the lists 190/146/144 initialised
    from 90/46/44, as the copies of vlamcc.F:533-546), each cycle
    lambda <- (dE/dT + (dZ/dT)^T lambda) / D (NEWT2, :756) with the pair
    symmetrisation of the amplitude solver, convergence on the largest element
    of the change (DRTSTS, :791) and the DIIS of the amplitude solver over the
    reference's vector L1 + L2(AB) + packed L2(AA) (DODIIS0, :812).

    Returns dict(res, dres, converged, ncycle, L1, L2 (reference convention),
    l1, l2 (this module's))."""
    import torch
    from .diis import ReferenceDIIS
    TB = TorchBlocks(B, torch)
    o, v = B.o, B.v
    t1t = torch.tensor(t1, dtype=torch.float64, requires_grad=True)
    t2t = torch.tensor(t2, dtype=torch.float64, requires_grad=True)
    g1, g2 = torch.autograd.grad(_energy(TB, t1t, t2t), [t1t, t2t])
    g1, g2 = g1.numpy(), g2.numpy()
    Z1, Z2 = ccsd.residual(TB, t1t, t2t)
    D1, D2 = TB.Dov.detach().numpy(), TB.Doovv.detach().numpy()

    def jtv(l1, l2):
        a, b = torch.autograd.grad([Z1, Z2], [t1t, t2t], [torch.tensor(l1), torch.tensor(l2)],
                                   retain_graph=True)
        return a.numpy(), b.numpy()

    L1, L2 = np.array(t1, dtype=float), ccsd.symmetrize_t2(np.array(t2, dtype=float))
    dii = ReferenceDIIS(exporder)
    hist = dict(res=[], dres=[])
    converged = False
    for icycle in range(1, maxcyc + 1):
        l1, l2 = lambda_from_reference(L1, L2)
        a, b = jtv(l1, l2)
        n1, n2 = lambda_to_reference((g1 + a) / D1, ccsd.symmetrize_t2((g2 + b) / D2))
        res, dres, ext = dii.step(icycle, ccsd.diis_vector(L1, L2), ccsd.diis_vector(n1, n2))
        hist["res"].append(res)
        hist["dres"].append(dres)
        if abs(res) < 10.0 ** (-cc_conv):
            converged = True
            break
        if ext is not None:
            L1, L2 = (x.copy() for x in ccsd.split_vector(ext, o, v))
        else:
            L1, L2 = n1, n2
    l1, l2 = lambda_from_reference(L1, L2)
    hist.update(converged=converged, ncycle=icycle, L1=L1, L2=L2, l1=l1, l2=l2)
    return hist


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
