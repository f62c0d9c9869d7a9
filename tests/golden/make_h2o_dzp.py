"""Generate the H2O molecular-orbital fixtures that pin the CCSD oracle.

Run in a container that holds the reference tree (it reads the DZP and
cc-pVDZ basis sets from the reference's basis library, test/KEEP/GENBAS, and
nothing else); the reference root is a required argument:

    python tests/golden/make_h2o_dzp.py <reference root> [tag ...]

Writes tests/golden/<file> for the geometries of the reference's regression
inputs and for the cc-pVDZ benchmark system:

  * ``zmat035``: test/zmat.035.ccsd (R=0.957 A, A=104.5 deg), DZP, golden CCSD
    iteration energies in test/OUTPUT/out.zmat.035.ccsd:555-650;
  * ``zmat020``: test/zmat.020 (R=1.0 A, A=104 deg), DZP, golden CCSD and (T)
    energies in test/OUTPUT/out.zmat.020:650-688;
  * ``zmat026``: test/zmat.026 (R=0.96 A, A=104 deg), DZP, CCSD first-order
    properties;
  * ``zmat046``: test/zmat.046 (R=0.95720197 A, A=104.52 deg), DZP with
    Cartesian d (SPHERICAL=OFF); the reference runs a UHF-CCSD on this closed
    shell, whose SCF, MP2 and converged CCSD energies equal the RHF ones
    (test/OUTPUT/out.zmat.046:461,605-608,745);
  * ``ccpvdz``: H2O at R=0.9572 A, A=104.52 deg in cc-pVDZ with spherical d
    functions (24 basis functions, 5 occupied / 19 virtual, C2v), the
    plain-FP64 benchmark system; the reference has no output for it, so it
    is pinned through the oracle only.

Each file holds: orbital energies (occupied then virtual, each block sorted by
irrep as the reference's DPD lists order them), the irrep populations
(pop, vrt), the MO two-electron integrals (pq|rs) packed with 8-fold symmetry,
the MO dipole and diagonal second-moment (x^2, y^2, z^2) integrals about the
origin (the centre of mass) with their nuclear counterparts, E(SCF) and the
nuclear repulsion energy.

Where the reference prints them, the SCF and nuclear repulsion energies must
reproduce its records; the script asserts that.
"""
from __future__ import annotations

import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from _gto import BOHR_ANGSTROM, Basis  # noqa: E402

GEOMS = {
    # tag: (R angstrom, angle deg, golden SCF energy, golden nuclear repulsion,
    #       GENBAS basis name, spherical d, number of basis functions, file)
    "zmat035": (0.957, 104.5, -76.0465033211, 9.19693438045,    # test/zmat.035.ccsd TEST.DAT
                "DZP", False, 26, "h2o_dzp_zmat035.npz"),
    "zmat020": (1.0, 104.0, -76.0407105174, 8.80260376799,      # test/zmat.020 TEST.DAT
                "DZP", False, 26, "h2o_dzp_zmat020.npz"),
    "zmat026": (0.96, 104.0, -76.0462837076, 9.16937892499,     # test/zmat.026 TEST.DAT
                "DZP", False, 26, "h2o_dzp_zmat026.npz"),
    "zmat046": (0.95720197, 104.52, -76.046493464757, 9.1949465922,  # out.zmat.046:339,605
                "DZP", False, 26, "h2o_dzp_zmat046.npz"),
    "ccpvdz": (0.9572, 104.52, None, None, "CC-PVDZ", True, 24, "h2o_ccpvdz.npz"),
}


def read_genbas(path, key):
    """Parse one GENBAS entry: returns list of (l, exps, coefs[nprim, ncontr])."""
    lines = open(path).read().splitlines()
    i = next(k for k, s in enumerate(lines) if s.strip() == key)
    i += 2
    while not lines[i].strip():
        i += 1
    nshell = int(lines[i].split()[0]); i += 1
    ls = [int(x) for x in lines[i].split()]; i += 1
    ncon = [int(x) for x in lines[i].split()]; i += 1
    nprim = [int(x) for x in lines[i].split()]; i += 1
    out = []
    vals = []
    for s in range(nshell):
        # exponents
        exps = []
        while len(exps) < nprim[s]:
            t = lines[i].split(); i += 1
            exps += [float(x) for x in t]
        coefs = []
        while len(coefs) < nprim[s] * ncon[s]:
            t = lines[i].split(); i += 1
            coefs += [float(x) for x in t]
        out.append((ls[s], np.array(exps), np.array(coefs).reshape(nprim[s], ncon[s])))
    del vals
    return out


def geometry(R_ang, A_deg):
    """O on the C2 (z) axis, H atoms in the xz plane (the reference's frame)."""
    R = R_ang / BOHR_ANGSTROM
    half = np.deg2rad(A_deg) / 2
    xh = R * np.sin(half)
    zh = R * np.cos(half)
    # put the centre of mass at the origin (irrelevant for energies; dipoles are
    # reported for the neutral molecule, origin independent)
    mO, mH = 15.99491461956, 1.00782503207
    zcom = (2 * mH * zh) / (mO + 2 * mH)
    O = np.array([0.0, 0.0, -zcom])
    H1 = np.array([xh, 0.0, zh - zcom])
    H2 = np.array([-xh, 0.0, zh - zcom])
    return [("O", 8.0, O), ("H", 1.0, H1), ("H", 1.0, H2)]


def nuclear_repulsion(atoms):
    e = 0.0
    for i in range(len(atoms)):
        for j in range(i):
            e += atoms[i][1] * atoms[j][1] / np.linalg.norm(atoms[i][2] - atoms[j][2])
    return e


def rhf(S, H, G, nocc, tol=1e-13, maxit=200):
    """Closed-shell Roothaan-Hall SCF with Pulay DIIS; returns (E_elec, eps, C)."""
    s, U = np.linalg.eigh(S)
    X = U @ np.diag(s ** -0.5) @ U.T
    e, Cp = np.linalg.eigh(X.T @ H @ X)
    C = X @ Cp
    focks, errs = [], []
    E_old = 0.0
    for it in range(maxit):
        Cocc = C[:, :nocc]
        Dm = Cocc @ Cocc.T
        J = np.einsum("pqrs,rs->pq", G, Dm)
        K = np.einsum("prqs,rs->pq", G, Dm)
        F = H + 2 * J - K
        E = np.sum(Dm * (H + F))
        err = F @ Dm @ S - S @ Dm @ F
        focks.append(F); errs.append(err)
        focks, errs = focks[-8:], errs[-8:]
        n = len(focks)
        if n > 1:
            B = -np.ones((n + 1, n + 1)); B[-1, -1] = 0
            for i in range(n):
                for j in range(n):
                    B[i, j] = np.sum(errs[i] * errs[j])
            rhs = np.zeros(n + 1); rhs[-1] = -1
            c = np.linalg.solve(B, rhs)[:n]
            F = sum(ci * Fi for ci, Fi in zip(c, focks))
        e, Cp = np.linalg.eigh(X.T @ F @ X)
        C = X @ Cp
        if abs(E - E_old) < tol and np.max(np.abs(err)) < 1e-10:
            break
        E_old = E
    # final diagonalisation of the converged (un-extrapolated) Fock matrix
    Cocc = C[:, :nocc]
    Dm = Cocc @ Cocc.T
    J = np.einsum("pqrs,rs->pq", G, Dm)
    K = np.einsum("prqs,rs->pq", G, Dm)
    F = H + 2 * J - K
    E = np.sum(Dm * (H + F))
    e, Cp = np.linalg.eigh(X.T @ F @ X)
    C = X @ Cp
    return E, e, C


def classify_irreps(basis, C, S):
    """Irrep (0..3 = A1, B2, B1, A2 in the reference's numbering) of each MO.

    Bit 0: odd under y -> -y; bit 1: odd under x -> -x.  With the molecule in
    the xz plane this gives A1=1, B2=2, B1=3, A2=4 (1-based), the reference's
    order (test/OUTPUT/out.zmat.035.ccsd, orbital table COMPSYM column).
    """
    cen = np.array(basis.ao_center)
    n = basis.nao
    # AO index of each function's mirror image
    def mirror(axis):
        R = np.zeros((n, n))
        # group AOs by centre, in generation order
        for mu in range(n):
            img = cen[mu].copy(); img[axis] = -img[axis]
            same = [nu for nu in range(n) if np.allclose(cen[nu], cen[mu], atol=1e-12)]
            mates = [nu for nu in range(n) if np.allclose(cen[nu], img, atol=1e-12)]
            k = same.index(mu)
            nu = mates[k]
            R[nu, mu] = (-1) ** basis.ao_l[mu][axis]
        return R
    My = mirror(1)
    Mx = mirror(0)
    irr = []
    for k in range(C.shape[1]):
        c = C[:, k]
        py = c @ S @ (My @ c)
        px = c @ S @ (Mx @ c)
        assert abs(abs(py) - 1) < 1e-8 and abs(abs(px) - 1) < 1e-8, (k, py, px)
        irr.append((0 if py > 0 else 1) | ((0 if px > 0 else 1) << 1))
    return np.array(irr)


def pack8(g):
    """Pack (pq|rs) with 8-fold symmetry: pq = p>=q, rs = r>=s, pq >= rs."""
    n = g.shape[0]
    tri = [(p, q) for p in range(n) for q in range(p + 1)]
    npair = len(tri)
    idx = np.array(tri)
    M = g[idx[:, 0][:, None], idx[:, 1][:, None], idx[:, 0][None, :], idx[:, 1][None, :]]
    iu = np.tril_indices(npair)
    return M[iu]


def build(ref_root, tag):
    R, A, e_scf_gold, enuc_gold, bname, spherical, nbf, fname = GEOMS[tag]
    genbas = os.path.join(ref_root, "test", "KEEP", "GENBAS")
    atoms = geometry(R, A)
    shells = []
    for sym, Z, xyz in atoms:
        for l, exps, coefs in read_genbas(genbas, f"{sym}:{bname}"):
            shells.append((xyz, l, exps, coefs))
    basis = Basis(shells, spherical=spherical)
    assert basis.nao == nbf, basis.nao
    S, T, V, Mu = basis.one_electron([a[1] for a in atoms], [a[2] for a in atoms])
    G = basis.eri()
    enuc = nuclear_repulsion(atoms)
    nocc = 5
    E_el, eps, C = rhf(S, T + V, G, nocc)
    E_scf = E_el + enuc
    print(f"{tag}: Enuc={enuc:.11f} (golden {enuc_gold}) E_SCF={E_scf:.10f} (golden {e_scf_gold})")
    if enuc_gold is not None:
        assert abs(enuc - enuc_gold) < 1e-9
    if e_scf_gold is not None:
        assert abs(E_scf - e_scf_gold) < 2e-10, E_scf - e_scf_gold
    irr = classify_irreps(basis, C, S)
    # reference DPD ordering: occupied by irrep, virtual by irrep, energy order within
    occ = [k for h in range(4) for k in range(nocc) if irr[k] == h]
    vir = [k for h in range(4) for k in range(nocc, basis.nao) if irr[k] == h]
    order = occ + vir
    C = C[:, order]; eps = eps[order]; irr = irr[order]
    pop = np.array([np.sum(irr[:nocc] == h) for h in range(4)])
    vrt = np.array([np.sum(irr[nocc:] == h) for h in range(4)])
    g = np.einsum("pqrs,pi->iqrs", G, C, optimize=True)
    g = np.einsum("iqrs,qj->ijrs", g, C, optimize=True)
    g = np.einsum("ijrs,rk->ijks", g, C, optimize=True)
    g = np.einsum("ijks,sl->ijkl", g, C, optimize=True)
    mu_mo = np.array([C.T @ Mu[d] @ C for d in range(3)])
    q_mo = np.array([C.T @ basis.second_moments[d] @ C for d in range(3)])
    nucsecond = sum(a[1] * a[2] ** 2 for a in atoms)
    charges = np.array([a[1] for a in atoms])
    nucdip = sum(a[1] * a[2] for a in atoms)
    h_mo = C.T @ (T + V) @ C
    np.savez_compressed(
        os.path.join(os.path.dirname(os.path.abspath(__file__)), fname),
        eps=eps, irrep=irr, pop=pop, vrt=vrt, eri8=pack8(g), nmo=basis.nao,
        dipole=mu_mo, nucdip=nucdip, second=q_mo, nucsecond=nucsecond, hcore=h_mo,
        e_scf=E_scf, e_nuc=enuc,
        charges=charges,
    )
    return eps, irr, pop, vrt, g


if __name__ == "__main__":
    if len(sys.argv) < 2:
        raise SystemExit("usage: make_h2o_dzp.py <reference root> [tag ...]")
    ref = sys.argv[1]
    tags = sys.argv[2:] or list(GEOMS)
    for tag in tags:
        build(ref, tag)
