"""Cartesian Gaussian integrals (McMurchie-Davidson) and RHF SCF, in numpy.

Test infrastructure only: this module builds the molecular-orbital Hamiltonians
that pin the CCSD oracle to the reference's golden outputs (H2O/DZP, Cartesian
d functions, C2v).  The reference produces the same quantities with its own
integral program (vmol/), SCF (vscf/) and transformation (vtran/, intprc/);
those are Fortran and are not buildable here, so the published McMurchie-
Davidson scheme is restated instead:

  * Hermite expansion coefficients E^{ij}_t (McMurchie & Davidson,
    J. Comput. Phys. 26, 218 (1978));
  * Hermite Coulomb integrals R^n_{tuv} from the Boys function;
  * closed-shell Roothaan-Hall SCF with Pulay DIIS.

Energies are invariant to the normalisation of contracted functions and to the
choice of real Cartesian components, so only the primitive exponents and the
contraction coefficients (which multiply normalised primitives, the GENBAS
convention) matter.
"""
from __future__ import annotations

import itertools
import math

import numpy as np
from scipy.special import gammainc, gammaln

BOHR_ANGSTROM = 0.529177249  # joda/angs2bohr.F:7


def cart_components(l):
    """Cartesian exponent triples of total degree l (xx, xy, xz, yy, yz, zz for d)."""
    out = []
    for lx in range(l, -1, -1):
        for ly in range(l - lx, -1, -1):
            out.append((lx, ly, l - lx - ly))
    return out


def boys(nmax, T):
    """F_n(T) for n = 0..nmax, T an array.  Returns shape (nmax+1,) + T.shape."""
    T = np.asarray(T, dtype=np.float64)
    out = np.empty((nmax + 1,) + T.shape)
    small = T < 1e-10
    Ts = np.where(small, 1.0, T)
    for n in range(nmax + 1):
        a = n + 0.5
        # F_n(T) = Gamma(n+1/2) P(n+1/2, T) / (2 T^{n+1/2})
        val = np.exp(gammaln(a)) * gammainc(a, Ts) / (2.0 * Ts ** a)
        # series for tiny T: F_n(T) = 1/(2n+1) - T/(2n+3)
        ser = 1.0 / (2 * n + 1) - T / (2 * n + 3)
        out[n] = np.where(small, ser, val)
    return out


def hermite_E(la, lb, a, b, XA, XB):
    """Hermite expansion coefficients for one Cartesian direction.

    a, b: exponent arrays (N,); XA, XB: coordinates (N,).  Returns E with shape
    (la+1, lb+1, la+lb+1, N): E[i, j, t] for the product x_A^i x_B^j gaussians.
    """
    p = a + b
    mu = a * b / p
    Xab = XA - XB
    P = (a * XA + b * XB) / p
    Xpa = P - XA
    Xpb = P - XB
    N = a.shape[0]
    E = np.zeros((la + 1, lb + 1, la + lb + 2, N))
    E[0, 0, 0] = np.exp(-mu * Xab * Xab)
    inv2p = 0.5 / p
    for i in range(la + 1):
        for j in range(lb + 1):
            if i == 0 and j == 0:
                continue
            if i > 0:
                src = E[i - 1, j]
                X = Xpa
            else:
                src = E[i, j - 1]
                X = Xpb
            for t in range(i + j + 1):
                v = X * src[t]
                if t > 0:
                    v = v + inv2p * src[t - 1]
                v = v + (t + 1) * src[t + 1]
                E[i, j, t] = v
    return E[:, :, : la + lb + 1]


def hermite_R(L, alpha, PC):
    """R_{tuv}(alpha, PC) for t+u+v <= L.  PC: (3, N).  Returns dict (t,u,v)->(N,)."""
    X, Y, Z = PC
    T = alpha * (X * X + Y * Y + Z * Z)
    F = boys(L, T)
    # R^n_{000}
    Rn = {}
    m2a = -2.0 * alpha
    for n in range(L + 1):
        Rn[(0, 0, 0, n)] = (m2a ** n) * F[n]
    for tot in range(1, L + 1):
        for n in range(L - tot + 1):
            for t in range(tot + 1):
                for u in range(tot - t + 1):
                    v = tot - t - u
                    if t > 0:
                        val = X * Rn[(t - 1, u, v, n + 1)]
                        if t > 1:
                            val = val + (t - 1) * Rn[(t - 2, u, v, n + 1)]
                    elif u > 0:
                        val = Y * Rn[(t, u - 1, v, n + 1)]
                        if u > 1:
                            val = val + (u - 1) * Rn[(t, u - 2, v, n + 1)]
                    else:
                        val = Z * Rn[(t, u, v - 1, n + 1)]
                        if v > 1:
                            val = val + (v - 1) * Rn[(t, u, v - 2, n + 1)]
                    Rn[(t, u, v, n)] = val
    return {(t, u, v): Rn[(t, u, v, 0)] for (t, u, v, n) in Rn if n == 0}


# Real solid harmonics of degree 2 as combinations of the normalised
# Cartesian components (xx, xy, xz, yy, yz, zz), each normalised by itself:
# with x^2 = sqrt(3) g_xx (up to the common radial norm) the five pure-d
# polynomials xy, xz, yz, x^2 - y^2, 2z^2 - x^2 - y^2 are spanned without the
# r^2 (s-type) combination.  Scale factors do not matter (energies are
# invariant to the normalisation of each AO).  The second entry is a
# representative exponent triple whose parities under x -> -x and y -> -y are
# the function's own (used to classify molecular orbitals by irrep).
_SPH_D = [
    ([0.0, 1.0, 0.0, 0.0, 0.0, 0.0], (1, 1, 0)),                 # xy
    ([0.0, 0.0, 1.0, 0.0, 0.0, 0.0], (1, 0, 1)),                 # xz
    ([0.0, 0.0, 0.0, 0.0, 1.0, 0.0], (0, 1, 1)),                 # yz
    ([math.sqrt(3.0), 0.0, 0.0, -math.sqrt(3.0), 0.0, 0.0], (2, 0, 0)),   # x^2 - y^2
    ([-math.sqrt(3.0), 0.0, 0.0, -math.sqrt(3.0), 0.0, 2.0 * math.sqrt(3.0)], (0, 0, 2)),
]


class Basis:
    """Primitive Cartesian functions and their contraction into AO functions.

    shells: list of (center(3,), l, exps(np), coefs(np, ncontr)) per atom shell
    block as read from GENBAS.  With ``spherical`` the d shells contribute the
    five real solid harmonics instead of the six Cartesian components (the
    reference's SPHERICAL=ON, its default for the correlation-consistent
    sets); s and p shells are the same either way.
    """

    def __init__(self, shells, spherical=False):
        self.prim_shells = []  # (center, l, alpha)
        self.prim_funcs = []   # (prim_shell_index, (lx,ly,lz))
        rows = []              # contraction entries (prim_func, ao, coef)
        nao = 0
        self.ao_center = []
        self.ao_l = []
        for center, l, exps, coefs in shells:
            comps = cart_components(l)
            ncontr = coefs.shape[1]
            pidx0 = len(self.prim_funcs)
            for k, alpha in enumerate(exps):
                self.prim_shells.append((np.asarray(center, float), l, float(alpha)))
                for c in comps:
                    self.prim_funcs.append((len(self.prim_shells) - 1, c))
            for ic in range(ncontr):
                for ci, c in enumerate(comps):
                    ao = nao + ic * len(comps) + ci
                    for k, alpha in enumerate(exps):
                        if coefs[k, ic] != 0.0:
                            # normalised primitive: (2a/pi)^{3/4} (4a)^{l/2} / sqrt(prod (2l_x-1)!!)
                            dfac = np.prod([_dfact(2 * x - 1) for x in c])
                            norm = (2 * alpha / math.pi) ** 0.75 * (4 * alpha) ** (l / 2) / math.sqrt(dfac)
                            rows.append((pidx0 + k * len(comps) + ci, ao, coefs[k, ic] * norm))
            for ic in range(ncontr):
                for ci, c in enumerate(comps):
                    self.ao_center.append(np.asarray(center, float))
                    self.ao_l.append(c)
            nao += ncontr * len(comps)
        self.nao = nao
        self.nprim = len(self.prim_funcs)
        D = np.zeros((self.nprim, nao))
        for p, ao, c in rows:
            D[p, ao] += c
        if spherical:
            # Cartesian AO -> spherical AO, shell by shell in generation order
            cols, centers, ls = [], [], []
            k = 0
            for center, l, exps, coefs in shells:
                ncomp = len(cart_components(l))
                for ic in range(coefs.shape[1]):
                    if l < 2:
                        for ci in range(ncomp):
                            e = np.zeros(nao); e[k + ci] = 1.0
                            cols.append(e)
                            centers.append(self.ao_center[k + ci]); ls.append(self.ao_l[k + ci])
                    elif l == 2:
                        for w, rep in _SPH_D:
                            e = np.zeros(nao); e[k:k + 6] = w
                            cols.append(e)
                            centers.append(self.ao_center[k]); ls.append(rep)
                    else:
                        raise NotImplementedError("spherical functions above d")
                    k += ncomp
            Tcs = np.array(cols).T
            D = D @ Tcs
            self.nao = Tcs.shape[1]
            self.ao_center, self.ao_l = centers, ls
        self.D = D

    # ---- primitive-level integrals, grouped by angular-momentum class ----
    def _shell_arrays(self, idx):
        cen = np.array([self.prim_shells[i][0] for i in idx])
        alp = np.array([self.prim_shells[i][2] for i in idx])
        return cen, alp

    def _by_l(self):
        groups = {}
        for i, (_, l, _) in enumerate(self.prim_shells):
            groups.setdefault(l, []).append(i)
        return groups

    def _func_index(self):
        # prim shell index -> list of prim func indices in component order
        m = {}
        for f, (s, c) in enumerate(self.prim_funcs):
            m.setdefault(s, []).append(f)
        return m

    def one_electron(self, charges, centers):
        """Overlap S, kinetic T, nuclear attraction V, and dipole moments (x,y,z) about origin;
        the diagonal second moments (x^2, y^2, z^2) are left in ``self.second_moments``."""
        groups = self._by_l()
        fidx = self._func_index()
        n = self.nprim
        S = np.zeros((n, n)); T = np.zeros((n, n)); V = np.zeros((n, n))
        M = np.zeros((3, n, n))
        Q = np.zeros((3, n, n))
        for la, ia in groups.items():
            for lb, ib in groups.items():
                pairs = list(itertools.product(ia, ib))
                A, a = self._shell_arrays([p[0] for p in pairs])
                B, b = self._shell_arrays([p[1] for p in pairs])
                p = a + b
                P = (a[:, None] * A + b[:, None] * B) / p[:, None]
                Ex = [hermite_E(la, lb + 2, a, b, A[:, d], B[:, d]) for d in range(3)]
                ca = cart_components(la)
                cb = cart_components(lb)
                sq = np.sqrt(np.pi / p)
                Rs = []
                L = la + lb
                for C in centers:
                    Rs.append(hermite_R(L, p, (P - np.asarray(C)[None, :]).T))
                for ci, (ax, ay, az) in enumerate(ca):
                    for cj, (bx, by, bz) in enumerate(cb):
                        e = [(ax, bx), (ay, by), (az, bz)]
                        s1 = [Ex[d][e[d][0], e[d][1], 0] * sq for d in range(3)]
                        # kinetic 1D: b(2j+1) S(i,j) - 2b^2 S(i,j+2) - j(j-1)/2 S(i,j-2)
                        t1 = []
                        for d in range(3):
                            i_, j_ = e[d]
                            val = b * (2 * j_ + 1) * Ex[d][i_, j_, 0] * sq
                            val = val - 2 * b * b * Ex[d][i_, j_ + 2, 0] * sq
                            if j_ >= 2:
                                val = val - 0.5 * j_ * (j_ - 1) * Ex[d][i_, j_ - 2, 0] * sq
                            t1.append(val)
                        sval = s1[0] * s1[1] * s1[2]
                        tval = t1[0] * s1[1] * s1[2] + s1[0] * t1[1] * s1[2] + s1[0] * s1[1] * t1[2]
                        vval = np.zeros_like(sval)
                        for Zc, R in zip(charges, Rs):
                            acc = np.zeros_like(sval)
                            for t in range(ax + bx + 1):
                                for u in range(ay + by + 1):
                                    for v in range(az + bz + 1):
                                        acc += (Ex[0][ax, bx, t] * Ex[1][ay, by, u]
                                                * Ex[2][az, bz, v] * R[(t, u, v)])
                            vval -= Zc * 2 * np.pi / p * acc
                        mvals = []
                        qvals = []
                        for d in range(3):
                            i_, j_ = e[d]
                            # <x_C> about origin: E_1 + P_x E_0
                            m1 = (Ex[d][i_, j_, 1] if i_ + j_ >= 1 else 0.0) + P[:, d] * Ex[d][i_, j_, 0]
                            m1 = m1 * sq
                            mvals.append(m1 * s1[(d + 1) % 3] * s1[(d + 2) % 3])
                            # <x^2> about origin: 2 E_2 + 2 P_x E_1 + (P_x^2 + 1/(2p)) E_0
                            m2 = ((2.0 * Ex[d][i_, j_, 2] if i_ + j_ >= 2 else 0.0)
                                  + (2.0 * P[:, d] * Ex[d][i_, j_, 1] if i_ + j_ >= 1 else 0.0)
                                  + (P[:, d] ** 2 + 0.5 / p) * Ex[d][i_, j_, 0]) * sq
                            qvals.append(m2 * s1[(d + 1) % 3] * s1[(d + 2) % 3])
                        for k, (sa, sb) in enumerate(pairs):
                            fa = fidx[sa][ci]
                            fb = fidx[sb][cj]
                            S[fa, fb] = sval[k]
                            T[fa, fb] = tval[k]
                            V[fa, fb] = vval[k]
                            for d in range(3):
                                M[d, fa, fb] = mvals[d][k]
                                Q[d, fa, fb] = qvals[d][k]
        D = self.D
        tr = lambda X: D.T @ X @ D
        # diagonal second moments <x^2>, <y^2>, <z^2> about the origin
        self.second_moments = np.array([tr(Q[d]) for d in range(3)])
        return tr(S), tr(T), tr(V), np.array([tr(M[d]) for d in range(3)])

    def eri(self):
        """Contracted AO electron-repulsion integrals (mu nu|lam sig), chemists' notation."""
        groups = self._by_l()
        fidx = self._func_index()
        n = self.nprim
        G = np.zeros((n, n, n, n))
        ls = sorted(groups)
        pair_data = {}
        for la in ls:
            for lb in ls:
                pairs = list(itertools.product(groups[la], groups[lb]))
                A, a = self._shell_arrays([p[0] for p in pairs])
                B, b = self._shell_arrays([p[1] for p in pairs])
                p = a + b
                P = (a[:, None] * A + b[:, None] * B) / p[:, None]
                Ex = [hermite_E(la, lb, a, b, A[:, d], B[:, d]) for d in range(3)]
                coef = {}
                for ci, (ax, ay, az) in enumerate(cart_components(la)):
                    for cj, (bx, by, bz) in enumerate(cart_components(lb)):
                        d = {}
                        for t in range(ax + bx + 1):
                            for u in range(ay + by + 1):
                                for v in range(az + bz + 1):
                                    d[(t, u, v)] = Ex[0][ax, bx, t] * Ex[1][ay, by, u] * Ex[2][az, bz, v]
                        coef[(ci, cj)] = d
                ia = np.array([fidx[s[0]] for s in pairs])
                ib = np.array([fidx[s[1]] for s in pairs])
                pair_data[(la, lb)] = (p, P, coef, ia, ib)
        for (la, lb), (p, P, cab, ia, ib) in pair_data.items():
            tuv_ab = sorted({k for d in cab.values() for k in d})
            for (lc, ld), (q, Q, ccd, ic, id_) in pair_data.items():
                L = la + lb + lc + ld
                pp = p[:, None]
                qq = q[None, :]
                alpha = pp * qq / (pp + qq)
                PQ = P[:, None, :] - Q[None, :, :]
                R = hermite_R(L, alpha.ravel(), PQ.reshape(-1, 3).T)
                shape = alpha.shape
                R = {k: v.reshape(shape) for k, v in R.items()}
                pref = 2 * np.pi ** 2.5 / (pp * qq * np.sqrt(pp + qq))
                for (ck, cl), dcd in ccd.items():
                    inner = {}
                    for (t, u, v) in tuv_ab:
                        acc = np.zeros(shape)
                        for (tt, uu, vv), ecd in dcd.items():
                            sgn = -1.0 if (tt + uu + vv) % 2 else 1.0
                            acc += sgn * ecd[None, :] * R[(t + tt, u + uu, v + vv)]
                        inner[(t, u, v)] = acc
                    for (ci, cj), dab in cab.items():
                        acc = np.zeros(shape)
                        for k, eab in dab.items():
                            acc += eab[:, None] * inner[k]
                        G[ia[:, ci][:, None], ib[:, cj][:, None],
                          ic[:, ck][None, :], id_[:, cl][None, :]] = pref * acc
        D = self.D
        G = np.tensordot(G, D, axes=([0], [0]))
        G = np.tensordot(G, D, axes=([0], [0]))
        G = np.tensordot(G, D, axes=([0], [0]))
        G = np.tensordot(G, D, axes=([0], [0]))
        return G


def _dfact(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r
