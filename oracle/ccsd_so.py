"""Spin-orbital CCSD (Stanton, Gauss, Watts & Bartlett, J. Chem. Phys. 94,
4334 (1991)) -- oracle cross-check.

Test infrastructure: an independent, dense spin-orbital statement of the same
equations the reference's xvcc solves (the reference's own dense statement is
ccsd_light/ccsd_light_driver.F:226-540).  Used on small systems to validate
the spin-adapted closed-shell restatement in ``oracle.ccsd`` term by term,
including the non-Hartree-Fock Fock terms.
"""
from __future__ import annotations

import numpy as np


def _ct(spec, *ops):
    return np.einsum(spec, *ops, optimize=True)


def spin_hamiltonian(ham):
    """Antisymmetrised <PQ||RS> and Fock over spin orbitals.

    Spin-orbital order: occupied (i alpha, i beta) pairs, then virtual pairs;
    spin(P) = P % 2 within each block."""
    o, n = ham.nocc, ham.nmo
    spat = np.concatenate([np.repeat(np.arange(o), 2), np.repeat(np.arange(o, n), 2)])
    spin = np.tile([0, 1], n)
    # full spatial <pq|rs>
    full = np.zeros((n, n, n, n))
    for k1, s1 in (("o", slice(0, o)), ("v", slice(o, n))):
        for k2, s2 in (("o", slice(0, o)), ("v", slice(o, n))):
            for k3, s3 in (("o", slice(0, o)), ("v", slice(o, n))):
                for k4, s4 in (("o", slice(0, o)), ("v", slice(o, n))):
                    full[s1, s2, s3, s4] = ham.phys(k1 + k2 + k3 + k4)
    v = full[np.ix_(spat, spat, spat, spat)]
    sp = spin
    d13 = (sp[:, None, None, None] == sp[None, None, :, None])
    d24 = (sp[None, :, None, None] == sp[None, None, None, :])
    d14 = (sp[:, None, None, None] == sp[None, None, None, :])
    d23 = (sp[None, :, None, None] == sp[None, None, :, None])
    vp = v * (d13 & d24)
    vx = v.transpose(0, 1, 3, 2) * (d14 & d23)
    asym = vp - vx
    f = ham.fock[np.ix_(spat, spat)] * (sp[:, None] == sp[None, :])
    return asym, f, 2 * o


def to_spin_amplitudes(t1, t2):
    o, v = t1.shape
    so, sv = 2 * o, 2 * v
    sp_o = np.tile([0, 1], o)
    sp_v = np.tile([0, 1], v)
    io = np.repeat(np.arange(o), 2)
    iv = np.repeat(np.arange(v), 2)
    T1 = t1[np.ix_(io, iv)] * (sp_o[:, None] == sp_v[None, :])
    a = t2[np.ix_(io, io, iv, iv)]
    b = t2.transpose(0, 1, 3, 2)[np.ix_(io, io, iv, iv)]
    dIA = sp_o[:, None, None, None] == sp_v[None, None, :, None]
    dJB = sp_o[None, :, None, None] == sp_v[None, None, None, :]
    dIB = sp_o[:, None, None, None] == sp_v[None, None, None, :]
    dJA = sp_o[None, :, None, None] == sp_v[None, None, :, None]
    T2 = a * (dIA & dJB) - b * (dIB & dJA)
    return T1, T2


def residual(asym, f, no, T1, T2):
    """Stanton-Gauss eqs. (1)-(2) without the diagonal Fock terms: returns Z1, Z2
    with t = Z / D the Jacobi update."""
    o = slice(0, no)
    v = slice(no, asym.shape[0])
    fov = f[o, v]
    foo = f[o, o] - np.diag(np.diag(f[o, o]))
    fvv = f[v, v] - np.diag(np.diag(f[v, v]))
    oovv = asym[o, o, v, v]
    ooov = asym[o, o, o, v]
    ovvv = asym[o, v, v, v]
    taut = T2 + 0.5 * (_ct("ia,jb->ijab", T1, T1) - _ct("ib,ja->ijab", T1, T1))
    tau = T2 + _ct("ia,jb->ijab", T1, T1) - _ct("ib,ja->ijab", T1, T1)
    Fae = (fvv - 0.5 * _ct("me,ma->ae", fov, T1) + _ct("mf,mafe->ae", T1, ovvv)
           - 0.5 * _ct("mnaf,mnef->ae", taut, oovv))
    Fmi = (foo + 0.5 * _ct("ie,me->mi", T1, fov) + _ct("ne,mnie->mi", T1, ooov)
           + 0.5 * _ct("inef,mnef->mi", taut, oovv))
    Fme = fov + _ct("nf,mnef->me", T1, oovv)
    Wmnij = (asym[o, o, o, o] + _ct("je,mnie->mnij", T1, ooov)
             - _ct("ie,mnje->mnij", T1, ooov) + 0.25 * _ct("ijef,mnef->mnij", tau, oovv))
    Wabef = (asym[v, v, v, v] - _ct("mb,amef->abef", T1, asym[v, o, v, v])
             + _ct("ma,bmef->abef", T1, asym[v, o, v, v]) + 0.25 * _ct("mnab,mnef->abef", tau, oovv))
    Wmbej = (asym[o, v, v, o] + _ct("jf,mbef->mbej", T1, ovvv)
             - _ct("nb,mnej->mbej", T1, asym[o, o, v, o])
             - _ct("jnfb,mnef->mbej", 0.5 * T2 + _ct("jf,nb->jnfb", T1, T1), oovv))
    Z1 = (fov.copy() + _ct("ie,ae->ia", T1, Fae) - _ct("ma,mi->ia", T1, Fmi)
          + _ct("imae,me->ia", T2, Fme) - _ct("nf,naif->ia", T1, asym[o, v, o, v])
          - 0.5 * _ct("imef,maef->ia", T2, ovvv) - 0.5 * _ct("mnae,nmei->ia", T2, asym[o, o, v, o]))
    Z2 = oovv.copy()
    x = _ct("ijae,be->ijab", T2, Fae - 0.5 * _ct("mb,me->be", T1, Fme))
    Z2 += x - x.transpose(0, 1, 3, 2)
    x = _ct("imab,mj->ijab", T2, Fmi + 0.5 * _ct("je,me->mj", T1, Fme))
    Z2 -= x - x.transpose(1, 0, 2, 3)
    Z2 += 0.5 * _ct("mnab,mnij->ijab", tau, Wmnij)
    Z2 += 0.5 * _ct("ijef,abef->ijab", tau, Wabef)
    x = _ct("imae,mbej->ijab", T2, Wmbej) - _ct("ie,ma,mbej->ijab", T1, T1, asym[o, v, v, o])
    Z2 += x - x.transpose(1, 0, 2, 3) - x.transpose(0, 1, 3, 2) + x.transpose(1, 0, 3, 2)
    x = _ct("ie,abej->ijab", T1, asym[v, v, v, o])
    Z2 += x - x.transpose(1, 0, 2, 3)
    x = _ct("ma,mbij->ijab", T1, asym[o, v, o, o])
    Z2 -= x - x.transpose(0, 1, 3, 2)
    return Z1, Z2


def energy(asym, f, no, T1, T2):
    o = slice(0, no)
    v = slice(no, asym.shape[0])
    tau = T2 + _ct("ia,jb->ijab", T1, T1) - _ct("ib,ja->ijab", T1, T1)
    return np.sum(f[o, v] * T1) + 0.25 * np.sum(asym[o, o, v, v] * tau)
