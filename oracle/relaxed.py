"""Orbital-relaxed CCSD one-particle density by the Z-vector method -- oracle
(test infrastructure).

The reference's xdens adds the orbital response to the correlated density:
it forms the orbital gradient X(a,i) of the CC Lagrangian from the I(a,i)
and I(i,a) intermediates (dens/vdens.F:1036-1101, "FORM X(A,I) REQUIRED FOR
SOLVING THE Z-VECTOR EQUATIONS"), solves the Z-vector equations within
CPHF theory (MAKDIA1 / MAKDIA1_4STD_NONCAN, dens/vdens.F:1102-1137; the
"iterative expansion of D(ai)" of its output) and adds Z to the
virtual-occupied block of the density (FRMFUL 'REL', :1178).  This module
restates the same three steps for a closed-shell (RHF) CCSD from the
Lagrangian directly, with torch autograd in place of the reference's
hand-derived intermediates:

  * X_ai = dL/dkappa_ai at fixed amplitudes and multipliers, where
    L = E(T; f, g) + lambda . r(T; f, g) (oracle.lambda_ad) and the MO
    integrals g and Fock matrix f (which carries the SCF density) follow an
    orbital rotation U = 1 + kappa - kappa^T, kappa in the virtual-occupied
    block (first order suffices for a derivative at kappa = 0; CCSD is
    invariant to occupied-occupied and virtual-virtual rotations);
  * A_(bj),(ai) = d f_bj / d kappa_ai, the RHF response of the Brillouin
    condition f_ai = 0 (the SCF stationarity the Z multipliers enforce);
  * Z solves Z^T A = -X, and for a one-electron perturbation h -> h + x O
    the relaxed derivative is
        dE/dx = 2 sum_i O_ii + Tr(D O) + sum_bj Z_bj O_bj,
    D the unrelaxed correlation density of oracle.lambda_ad.density
    (the SCF term, the fixed-orbital CC term, the orbital relaxation).

Works on full MO integrals (a fixture Hamiltonian with ``_eri``); small
molecules only.
"""
from __future__ import annotations

import numpy as np

from . import ccsd, lambda_ad


class _RotatedBlocks:
    """The integral and Fock blocks oracle.ccsd.residual reads, as torch
    functions of an orbital rotation of a closed-shell Hamiltonian."""

    def __init__(self, ham, kappa, torch):
        o, n = ham.nocc, ham.nmo
        self.o, self.v = o, n - o
        K = torch.zeros((n, n), dtype=torch.float64)
        K = K.index_put((torch.arange(o, n)[:, None], torch.arange(o)[None, :]), kappa)
        U = torch.eye(n, dtype=torch.float64) + K - K.T
        g = torch.tensor(ham._eri, dtype=torch.float64)          # (pq|rs)
        h = torch.tensor(ham.hcore, dtype=torch.float64)
        g = torch.einsum("pqrs,pa,qb,rc,sd->abcd", g, U, U, U, U)
        h = U.T @ h @ U
        f = (h + 2.0 * torch.einsum("pqkk->pq", g[:, :, :o, :o])
             - torch.einsum("pkkq->pq", g[:, :o, :o, :]))
        self.f = f
        O, V = slice(0, o), slice(o, n)
        phys = lambda a, b, c, d: g[a, c, b, d].permute(0, 2, 1, 3)  # <ab|cd> = (ac|bd)
        self.oooo = phys(O, O, O, O)
        self.ooov = phys(O, O, O, V)
        self.oovv = phys(O, O, V, V)
        self.ovvo = phys(O, V, V, O)
        self.ovov = phys(O, V, O, V)
        self.ovvv = phys(O, V, V, V)
        self.vvvv = phys(V, V, V, V)
        self.foo, self.fvv, self.fov = f[O, O], f[V, V], f[O, V]
        self.eo = torch.diagonal(self.foo)
        self.ev = torch.diagonal(self.fvv)
        self.Dov = self.eo[:, None] - self.ev[None, :]
        self.Doovv = (self.eo[:, None, None, None] + self.eo[None, :, None, None]
                      - self.ev[None, None, :, None] - self.ev[None, None, None, :])


def orbital_gradient(ham, t1, t2, l1, l2):
    """X[a, i] = dL/dkappa_ai at kappa = 0 (the reference's X(a,i),
    dens/vdens.F:1087-1096), L the CC Lagrangian at the given converged
    amplitudes and multipliers (oracle.lambda_ad convention)."""
    import torch
    o, v = ham.nocc, ham.nvir
    kappa = torch.zeros((v, o), dtype=torch.float64, requires_grad=True)
    RB = _RotatedBlocks(ham, kappa, torch)
    T = lambda x: torch.tensor(np.asarray(x), dtype=torch.float64)
    t1t, t2t = T(t1), T(t2)
    r1, r2 = lambda_ad._r(RB, t1t, t2t)
    L = lambda_ad._energy(RB, t1t, t2t) + torch.sum(T(l1) * r1) + torch.sum(T(l2) * r2)
    (X,) = torch.autograd.grad(L, kappa)
    return X.numpy()


def brillouin_response(ham):
    """A[(b,j), (a,i)] = d f_bj / d kappa_ai at kappa = 0: the RHF orbital
    response the Z-vector equations invert (CPHF, dens/vdens.F:1102-1137)."""
    import torch
    o, v = ham.nocc, ham.nvir

    def fvo(kappa):
        return _RotatedBlocks(ham, kappa, torch).f[o:, :o]

    A = torch.autograd.functional.jacobian(fvo, torch.zeros((v, o), dtype=torch.float64))
    return A.reshape(v * o, v * o).numpy()


def relaxed_density(ham, cc_conv=11, maxcyc=200):
    """Converged CCSD and Lambda of a fixture Hamiltonian, then the Z-vector:
    returns dict(D (unrelaxed correlation density, oracle.lambda_ad.density),
    Z (v x o orbital-relaxation multipliers), X (orbital gradient), e_ccsd)."""
    r = ccsd.run_ccsd(ham, cc_conv=cc_conv, maxcyc=maxcyc, exporder=5)
    B = ccsd.Blocks(ham)
    lam = lambda_ad.iterate_lambda(B, r["t1"], r["t2"], cc_conv=cc_conv, maxcyc=maxcyc)
    if not r["converged"] or not lam["converged"]:
        raise RuntimeError("relaxed_density: CCSD or Lambda did not converge")
    D = lambda_ad.density(B, r["t1"], r["t2"], lam["l1"], lam["l2"])
    X = orbital_gradient(ham, r["t1"], r["t2"], lam["l1"], lam["l2"])
    A = brillouin_response(ham)
    Z = np.linalg.solve(A.T, -X.reshape(-1)).reshape(X.shape)
    return dict(D=D, Z=Z, X=X, e_ccsd=r["e_final"])


def property_derivative(ham, dens, O):
    """dE/dx for h -> h + x O (O symmetric, MO basis): the SCF, unrelaxed CC
    and orbital-relaxation terms, and their sum."""
    o = ham.nocc
    scf = 2.0 * np.trace(O[:o, :o])
    cc = float(np.sum(dens["D"] * O))
    relax = float(np.sum(dens["Z"] * O[o:, :o]))
    return dict(scf=scf, cc=cc, relax=relax, total=scf + cc + relax)
