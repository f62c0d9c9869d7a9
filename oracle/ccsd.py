"""Closed-shell (RHF) CCSD, restated from the reference's xvcc -- oracle.

Test infrastructure: the FP64 CPU restatement the CUDA engine is checked
against, and the timed CPU baseline.  Amplitudes use the reference's RHF
storage: only the alpha-beta doubles t2[i,j,a,b] = t_{iJ}^{aB} (list 46,
Ab x Ij) and alpha singles t1[i,a] (list 90); the same-spin doubles are
derived, t2(AA) = t2 - t2^T (libr2/abtoaa.F), exactly as the reference does
after every DIIS step (vcc/dodiis0.F:228).

The residual is the spin-integrated form of the Stanton-Gauss CCSD equations
that the reference's term routines implement; each block below names the
reference routine whose contribution it reproduces (call order of
vcc/vcc.F:811-1024).  Intermediates are spin-free closed-shell quantities;
"ABAB"/"ABBA" name the two spin blocks of W(mbej) that the RHF code keeps
(vcc/dwmbej.F, lists 54/56/58).

Integrals are physicists' notation v[p,q,r,s] = <pq|rs>.
"""
from __future__ import annotations

import numpy as np

from .diis import ReferenceDIIS


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _ct(spec, a, b):
    if _is_torch(a) or _is_torch(b):
        import torch
        return torch.einsum(spec, a, b)
    return np.einsum(spec, a, b, optimize=True)


def _tr(x, *axes):
    return x.permute(*axes) if _is_torch(x) else x.transpose(*axes)


def _diag(x):
    if _is_torch(x):
        import torch
        return torch.diag(x)
    return np.diag(x)


def _copy(x):
    return x.clone() if _is_torch(x) else x.copy()


def _P(x):
    """P(ia,jb) X = X_ijab + X_jiba: the permutation that RHF spin adaptation
    reduces P(ij)P(ab) to for the alpha-beta block."""
    return x + _tr(x, 1, 0, 3, 2)


class Blocks:
    """The integral lists one CCSD iteration reads (intprc/clmoio.F map)."""

    def __init__(self, ham):
        o = ham.nocc
        f = ham.fock
        self.o, self.v = o, ham.nvir
        self.foo = f[:o, :o].copy()
        self.fvv = f[o:, o:].copy()
        self.fov = f[:o, o:].copy()
        self.eo = np.diag(self.foo).copy()
        self.ev = np.diag(self.fvv).copy()
        self.oooo = ham.phys("oooo")   # <mn|ij>   list 13
        self.ooov = ham.phys("ooov")   # <mn|ie>   lists 7-10
        self.oovv = ham.phys("oovv")   # <mn|ef>   list 16 (and resorts 17-22)
        self.ovvo = ham.phys("ovvo")   # <mb|ej>   list 25/26
        self.ovov = ham.phys("ovov")   # <mb|je>   list 23/24
        self.ovvv = ham.phys("ovvv")   # <ma|ef>   lists 27-30
        self.vvvv = ham.phys("vvvv")   # <ab|ef>   list 233
        self.Dov = self.eo[:, None] - self.ev[None, :]
        self.Doovv = (self.eo[:, None, None, None] + self.eo[None, :, None, None]
                      - self.ev[None, None, :, None] - self.ev[None, None, None, :])


def mp2_guess(B):
    """Initial amplitudes: T2 = <ij|ab>/D, T1 = 0 (intprc FORMT2 / vcc/drdtgss.F
    without a TGUESS file)."""
    t1 = np.zeros((B.o, B.v))
    t2 = B.oovv / B.Doovv
    return t1, t2


def tau(t1, t2, fac=1.0):
    """FTAU (libr/ftau.f): tau(ab,ij) = t2 + fac * t1(ai) t1(bj) (AB spin case)."""
    return t2 + fac * _ct("ia,jb->ijab", t1, t1)


def energy(B, t1, t2):
    """CMPENG/TENER (libr/cmpeng.F:102-181): returns (E_AA, E_AB, E_total).

    E_AB = sum tau <ij|ab>; E_AA (alpha-alpha only, as printed) =
    1/2 sum tau (<ij|ab> - <ij|ba>); E_total = 2 E_AA + E_AB (+ 2 f_ia t_ia,
    non-zero only for a non-Hartree-Fock reference)."""
    tt = tau(t1, t2)
    eab = np.sum(tt * B.oovv)
    eaa = 0.5 * np.sum(tt * (B.oovv - B.oovv.transpose(0, 1, 3, 2)))
    e1 = 2.0 * np.sum(B.fov * t1)
    return eaa, eab, 2.0 * eaa + eab + e1


def intermediates(B, t1, t2):
    """GENINT (vcc/genint.F:1-480): the F and W intermediates of one iteration."""
    o, v = B.o, B.v
    taut = tau(t1, t2, 0.5)
    tt = tau(t1, t2)
    L_oovv = 2.0 * B.oovv - _tr(B.oovv, 0, 1, 3, 2)      # 2<mn|ef>-<mn|fe>
    L_ovvv = 2.0 * B.ovvv - _tr(B.ovvv, 0, 1, 3, 2)      # L[m,a,f,e] = 2<ma|fe>-<ma|ef>
    L_ooov = 2.0 * B.ooov - _tr(B.ooov, 1, 0, 2, 3)      # 2<mn|ie>-<nm|ie>
    offv = B.fvv - _diag(B.ev)
    offo = B.foo - _diag(B.eo)
    # QUAD3 + T1RING(F(ae) part) + fock terms (vcc/quad3.f, libr/t1ring.F)
    Fae = (offv - 0.5 * _ct("me,ma->ae", B.fov, t1)
           + _ct("mf,mafe->ae", t1, L_ovvv)
           - _ct("mnaf,mnef->ae", taut, L_oovv))
    # QUAD2 + T1INW2(F(mi) part) (vcc/quad2.f, vcc/t1inw2.f)
    Fmi = (offo + 0.5 * _ct("ie,me->mi", t1, B.fov)
           + _ct("ne,mnie->mi", t1, L_ooov)
           + _ct("inef,mnef->mi", taut, L_oovv))
    # MAKFME (vcc/makfme.F)
    Fme = B.fov + _ct("nf,mnef->me", t1, L_oovv)
    # QUAD1 + T1INW2 (W(mnij), vcc/quad1.f, vcc/t1inw2.f); the whole
    # tau*tau*<mn|ef> product is folded into the hole-hole ladder.
    Wmnij = (B.oooo + _ct("je,mnie->mnij", t1, B.ooov)
             + _ct("ie,nmje->mnij", t1, B.ooov)
             + _ct("ijef,mnef->mnij", tt, B.oovv))
    # DWMBEJ + T1RING (vcc/dwmbej.F): W(mbej) ABAB and ABBA spin blocks
    Xn = 0.5 * t2 + _ct("jf,nb->jnfb", t1, t1)           # (1/2 t2 + t1 t1)[j,n,f,b]
    W_abab = (B.ovvo + _ct("jf,mbef->mbej", t1, B.ovvv)
              - _ct("nb,mnej->mbej", t1, _tr(B.ooov, 1, 0, 3, 2))   # <mn|ej> = <nm|je>
              - _ct("jnfb,mnef->mbej", Xn, B.oovv)
              + _ct("njfb,mnef->mbej", t2, B.oovv)
              - 0.5 * _ct("njfb,mnfe->mbej", t2, B.oovv))
    # W_abba[m,b,e,j] (m alpha, b beta, e beta, j alpha)
    W_abba = (-_tr(B.ovov, 0, 1, 3, 2)
              - _ct("jf,mbfe->mbej", t1, B.ovvv)
              + _ct("nb,mnje->mbej", t1, B.ooov)
              + _ct("jnfb,mnfe->mbej", Xn, B.oovv))
    return dict(Fae=Fae, Fmi=Fmi, Fme=Fme, Wmnij=Wmnij, W_abab=W_abab, W_abba=W_abba,
                tau=tt)


def residual(B, t1, t2):
    """One pass of the xvcc term sequence (vcc/vcc.F:811-986): returns the
    T1 and T2 increments Z1, Z2 (everything except the diagonal Fock terms),
    so that the Jacobi update is t = Z / D (E4SENG / NEWT2)."""
    I = intermediates(B, t1, t2)
    Fae, Fmi, Fme = I["Fae"], I["Fmi"], I["Fme"]
    tt = I["tau"]
    # INITIN (vcc/initin.f): Z2 <- <ij|ab>;  INITSN: Z1 <- f(ia)
    Z2 = _copy(B.oovv)
    Z1 = _copy(B.fov)
    # FEACONT (vcc/feacont.f): P(ab) sum_e t(ij,ae)[F(be) - 1/2 t(mb)F(me)]; T1 += t(ie)F(ae)
    Fp = Fae - 0.5 * _ct("mb,me->be", t1, Fme)
    Z2 += _P(_ct("ijae,be->ijab", t2, Fp))
    Z1 += _ct("ie,ae->ia", t1, Fae)
    # FMICONT (vcc/fmicont.f): -P(ij) sum_m t(im,ab)[F(mj) + 1/2 t(je)F(me)]; T1 -= t(ma)F(mi)
    Fpp = Fmi + 0.5 * _ct("je,me->mj", t1, Fme)
    Z2 -= _P(_ct("imab,mj->ijab", t2, Fpp))
    Z1 -= _ct("ma,mi->ia", t1, Fmi)
    # FMECONT (vcc/fmecont.f): T1 += sum_me (2 t(im,ae) - t(mi,ae)) F(me)
    u = 2.0 * t2 - _tr(t2, 1, 0, 2, 3)
    Z1 += _ct("imae,me->ia", u, Fme)
    # T1INT2A (vcc/t1int2a.f): -P(ab) sum_m t(ma) <mb|ij>
    Z2 -= _P(_ct("ma,mbij->ijab", t1, _ovoo(B)))
    # T1INT2B (vcc/t1int2b.f): +P(ij) sum_e t(ie) <ab|ej>
    Z2 += _P(_ct("ie,abej->ijab", t1, _vvvo(B)))
    # T1INT1 (vcc/t1int1.F): T1 += sum_nf t(nf) (2<na|fi> - <na|if>)
    Z1 += _ct("nf,nafi->ia", t1, 2.0 * B.ovvo - _tr(B.ovov, 0, 1, 3, 2))
    # DRE3EN -> DRLAD (vcc/drlad.f, vcc/ladab1.F): hole-hole ladder sum_mn tau(mn,ab) W(mn,ij)
    Z2 += _ct("mnab,mnij->ijab", tt, I["Wmnij"])
    # DRLAD ITYPE=6: particle-particle ladder sum_ef <ab|ef> tau(ef,ij) (list 233)
    Z2 += _ct("ijef,abef->ijab", tt, B.vvvv)
    # T1INW1 (vcc/t1inw1.f): -P(ab) sum_m t(ma) [sum_ef <mb|ef> tau(ij,ef)]
    Zmbij = _ct("mbef,ijef->mbij", B.ovvv, tt)
    Z2 -= _P(_ct("ma,mbij->ijab", t1, Zmbij))
    # T12INT2 (vcc/t12int2.F): -P(ij)P(ab) sum_me t(ie) t(ma) <mb|ej>
    Z2 -= _P(_ct("imea,mbej->ijab", _ct("ie,ma->imea", t1, t1), B.ovvo)
             + _ct("jmea,mbie->ijab", _ct("je,ma->jmea", t1, t1), B.ovov))
    # DRRNG -> RNGDRV (vcc/drrng.f, vcc/rngdrv.f): ring terms with the ABAB
    # and ABBA W(mbej), symmetrised by SUMRNG
    Wab, Wba = I["W_abab"], I["W_abba"]
    ring = (_ct("imae,mbej->ijab", u, Wab)
            + _ct("imae,mbej->ijab", t2, Wba)
            + _ct("mjae,mbei->ijab", t2, Wba))
    Z2 += _P(ring)
    # E4S -> T2T1AB1/T2T1AB2 (vcc/e4s.F, libr/t2t1ab1.f, libr/t2t1ab2.f)
    w = 2.0 * t2 - _tr(t2, 0, 1, 3, 2)
    Z1 += _ct("imfe,maef->ia", w, B.ovvv)
    Z1 -= _ct("mnae,mnie->ia", u, B.ooov)
    return Z1, Z2


def ladder_packed(vvvv, tt):
    """The particle-particle ladder sum_ef <ab|ef> tau(ij,ef) in the RHF a<=b
    packing of vcc/ladab1.F:55-64 (pair blocks + SYMEXP4), in the symmetric /
    antisymmetric form the engine evaluates: with <ba|dc> = <ab|cd> and
    tau(ji,dc) = tau(ij,cd),
      U+[ab,cd] = (<ab|cd> + <ab|dc>)/2 (c<d), <ab|cc> (c=d);  tau+ = tau[cd] + tau[dc] (c<d), tau[cc]
      U-[ab,cd] = (<ab|cd> - <ab|dc>)/2 (c<d);                 tau- = tau[cd] - tau[dc]
      S[ij,a<=b] = sum_{c<=d} U+ tau+,  A[ij,a<b] = sum_{c<d} U- tau-
      Z[ab] = S + A,  Z[ba] = S - A,  Z[aa] = S.
    Returns Z[i,j,a,b] (the dense contraction's value)."""
    o, v = tt.shape[0], tt.shape[2]
    iu, ju = np.triu_indices(v)          # pairs c <= d (upper triangle incl. diagonal)
    im, jm = np.triu_indices(v, 1)       # pairs c < d
    diag = iu == ju
    Up = 0.5 * (vvvv[:, :, iu, ju] + vvvv[:, :, ju, iu])
    Up = Up[iu, ju]                      # rows a <= b
    Um = 0.5 * (vvvv[:, :, im, jm] - vvvv[:, :, jm, im])[im, jm]
    tp = tt[:, :, iu, ju] + tt[:, :, ju, iu]
    tp[:, :, diag] *= 0.5                # the diagonal pair once
    tm = tt[:, :, im, jm] - tt[:, :, jm, im]
    S = np.einsum("ijq,pq->ijp", tp, Up, optimize=True)
    A = np.einsum("ijq,pq->ijp", tm, Um, optimize=True)
    Z = np.zeros((o, o, v, v))
    Z[:, :, iu, ju] += S
    Z[:, :, ju, iu] += S * (~diag)       # Z[ba] = S - A below; the diagonal once
    Z[:, :, im, jm] += A
    Z[:, :, jm, im] -= A
    return Z


def _ovoo(B):
    """<mb|ij> as [m,b,i,j]; with real orbitals <mb|ij> = <ij|mb> = ooov[i,j,m,b]."""
    return _tr(B.ooov, 2, 3, 0, 1)


def _vvvo(B):
    """<ab|ej> as [a,b,e,j]: <ab|ej> = <ej|ab> = <je|ba> = ovvv[j,e,b,a]."""
    return _tr(B.ovvv, 3, 2, 1, 0)


def update(B, t1, t2):
    """E4SENG + NEWT2 (vcc/e4seng.F:150, libr2/newt2.F:244): divide the
    increments by the orbital-energy denominators (FP64)."""
    Z1, Z2 = residual(B, t1, t2)
    return Z1 / B.Dov, Z2 / B.Doovv


def diis_vector(t1, t2):
    """The DIIS vector of vcc/dodiis0.F:60-86 for RHF: T1(alpha), T2(AB) and
    the packed same-spin T2(AA) (a<b, i<j)."""
    o, v = t1.shape
    aa = t2 - t2.transpose(0, 1, 3, 2)
    ii, jj = np.triu_indices(o, 1)
    aa_p = aa[ii, jj][:, np.triu_indices(v, 1)[0], np.triu_indices(v, 1)[1]]
    return np.concatenate([t1.ravel(), t2.ravel(), aa_p.ravel()])


def split_vector(vec, o, v):
    n1 = o * v
    t1 = vec[:n1].reshape(o, v)
    t2 = vec[n1:n1 + o * o * v * v].reshape(o, o, v, v)
    return t1, t2


def symmetrize_t2(t2):
    """SYMETRIZE_T2 (vcc/dodiis0.F:57): t(ab,ij) <- (t(ab,ij) + t(ba,ji))/2."""
    return 0.5 * (t2 + t2.transpose(1, 0, 3, 2))


def run_ccsd(ham, cc_conv=7, maxcyc=50, exporder=5, t_guess=None, log=None,
             diis=True, damp=1.0):
    """The xvcc CC loop (vcc/vcc.F:797-1437) with DIIS (IFLAGS(21)=1).

    ``damp`` is DAMP_CC (IFLAGS2 damp_cc x 0.01, vcc/vcc.F:71): after NEWT2
    the new amplitudes become T_old + damp (T_new - T_old)
    (vcc/damp_cc_residual.F, called vcc/vcc.F:1031-1033, on the pair-
    symmetrised T2), the energy and the DIIS error vector are those of the
    damped amplitudes, and convergence is judged on the undamped difference,
    max |T_new - T_old|, i.e. the damped one divided by damp
    (vcc/dodiis0.F:93-97,165).  ``t_guess`` (t1, t2) replaces the MP2 start
    (the TGUESS restart, vcc/drdtgss.F).

    Returns a dict with the per-iteration energies (as printed by CMPENG on
    the new amplitudes), the residual and DIIS-residual maxima, the converged
    amplitudes and the final energy (CMPENG of the last accepted amplitudes,
    vcc/vcc.F:1101)."""
    B = Blocks(ham)
    t1, t2 = mp2_guess(B) if t_guess is None else t_guess
    e0 = energy(B, t1, t2)
    hist = dict(energies=[e0[2]], e_aa=[e0[0]], e_ab=[e0[1]], res=[], dres=[])
    dii = ReferenceDIIS(exporder)
    tol = 10.0 ** (-cc_conv)
    converged = False
    for icycle in range(1, maxcyc + 1):
        n1, n2 = update(B, t1, t2)
        n2 = symmetrize_t2(n2)
        t2s = symmetrize_t2(t2)
        if damp != 1.0:
            n1 = t1 + damp * (n1 - t1)
            n2 = t2s + damp * (n2 - t2s)
        eaa, eab, etot = energy(B, n1, n2)
        hist["energies"].append(etot); hist["e_aa"].append(eaa); hist["e_ab"].append(eab)
        if diis:
            x_old = diis_vector(t1, t2s)
            x_new = diis_vector(n1, n2)
            res, dres, ext = dii.step(icycle, x_old, x_new)
        else:
            d = diis_vector(n1, n2) - diis_vector(t1, t2s)
            res = d[np.argmax(np.abs(d))]
            dres, ext = res, None
        if damp != 1.0:
            res = res / damp
        hist["res"].append(res); hist["dres"].append(dres)
        if log:
            log(f"iter {icycle:3d}  E = {etot:.12f}  res = {res: .8e}  dres = {dres: .8e}")
        if abs(res) < tol:
            converged = True
            break
        if ext is not None:
            t1, t2 = split_vector(ext, B.o, B.v)
            t1 = t1.copy(); t2 = t2.copy()
        else:
            t1, t2 = n1, n2
    efinal = energy(B, t1, t2)
    hist.update(t1=t1, t2=t2, e_final=efinal[2], converged=converged, ncycle=icycle,
                blocks=B)
    return hist
