"""Host-side DPD (irrep-blocked) list packing over the engine's C-ABI.

A list with row pair type L and column pair type R stores, for every column
irrep h, an IRPDPD(h,L) x IRPDPD(h,R) column-major matrix (libr/inipck.F).
Pair indices come from the library's own ISYMOFF table
(acescore/aces_com_symloc.F): FULL pairs (p,q) sit at off + p + q*n_p, PACK
(p<q) pairs at off + p + q(q-1)/2 inside a diagonal irrep block, PCK2 (p<=q) at
off + p + q(q+1)/2.  Elements of antisymmetric PACK lists that are stored with
swapped indices carry a minus sign.
"""
from __future__ import annotations

import numpy as np

# pair types 1..25: (left space, right space, packing 0 FULL / 1 PACK / 2 PCK2)
_P = "VVOOVVOOVVVVVOVOOOVVOOVOO"
_Q = "VVOOVVOOOOOOVOVVVVVVOOVOV"


def pair_kind(t):
    return _P[t - 1], _Q[t - 1], (1 if t <= 4 else 2 if t <= 8 else 0)


class DPD:
    def __init__(self, lib, irr_o, irr_v):
        self.lib = lib
        self.nirrep = lib.nirrep
        self.irr = {"O": np.asarray(irr_o, dtype=np.int64), "V": np.asarray(irr_v, dtype=np.int64)}
        self.loc = {}
        self.cnt = {}
        for c, irr in self.irr.items():
            loc = np.zeros(len(irr), dtype=np.int64)
            cnt = np.zeros(8, dtype=np.int64)
            for k, h in enumerate(irr):
                loc[k] = cnt[h]
                cnt[h] += 1
            self.loc[c] = loc
            self.cnt[c] = cnt
        self._tables = {}

    def table(self, t):
        """(idx, sign, hpq) over all orbital pairs (p,q) of pair type t.

        idx: 0-based row/column index inside the irrep block hpq, -1 if the
        pair is not stored; sign: 1 canonical, -1 stored swapped with a sign
        change (PACK, antisymmetric), 2 stored swapped unchanged (PCK2), 0
        absent."""
        if t in self._tables:
            return self._tables[t]
        cp, cq, pk = pair_kind(t)
        ip, iq = self.irr[cp], self.irr[cq]
        lp, lq = self.loc[cp], self.loc[cq]
        npq = (len(ip), len(iq))
        idx = -np.ones(npq, dtype=np.int64)
        sgn = np.zeros(npq, dtype=np.int8)
        hpq = ip[:, None] ^ iq[None, :]
        off = np.zeros((8, 8), dtype=np.int64)
        for hq in range(self.nirrep):
            for h in range(self.nirrep):
                off[hq, h] = self.lib.isymoff(hq + 1, h + 1, t) - 1
        nump = self.cnt[cp]
        HP, HQ = np.meshgrid(ip, iq, indexing="ij")
        LP, LQ = np.meshgrid(lp, lq, indexing="ij")
        if pk == 0:
            idx = off[HQ, hpq] + LP + LQ * nump[HP]
            sgn[:] = 1
        else:
            canon = (HP < HQ) | ((HP == HQ) & (LP < LQ) if pk == 1 else (HP == HQ) & (LP <= LQ))
            swap = (HP > HQ) | ((HP == HQ) & (LP > LQ))
            tri = (lambda q: q * (q - 1) // 2) if pk == 1 else (lambda q: q * (q + 1) // 2)
            def index(hp, lp_, hq, lq_):
                rect = off[hq, hp ^ hq] + lp_ + lq_ * nump[hp]
                diag = off[hq, hp ^ hq] + lp_ + tri(lq_)
                return np.where(hp < hq, rect, diag)
            i1 = index(HP, LP, HQ, LQ)
            i2 = index(HQ, LQ, HP, LP)
            idx = np.where(canon, i1, np.where(swap, i2, -1))
            sgn = np.where(canon, 1, np.where(swap, -1 if pk == 1 else 2, 0)).astype(np.int8)
        self._tables[t] = (idx, sgn, hpq)
        return self._tables[t]


def _fast_c1(dpd, tl, tr):
    return dpd.nirrep == 1 and pair_kind(tl)[2] == 0 and pair_kind(tr)[2] == 0


def put_dense_list(lib, dpd, lst, tl, tr, dense):
    """PUTLST every irrep of list `lst` (types tl x tr) from dense[p,q,r,s]."""
    lib.inipck(1, tl, tr, lst)
    if _fast_c1(dpd, tl, tr):
        # row index p + q*np, column r + s*nr: the column-major matrix is the
        # fully transposed dense array
        buf = np.ascontiguousarray(np.asarray(dense, dtype=np.float64).transpose(3, 2, 1, 0))
        lib.putlst_raw(buf, 1, lib.irpdpd(1, tr), 1, lst)
        return
    ridx, rsgn, rh = dpd.table(tl)
    cidx, csgn, ch = dpd.table(tr)
    for h in range(dpd.nirrep):
        nr, nc = lib.irpdpd(h + 1, tl), lib.irpdpd(h + 1, tr)
        if nr == 0 or nc == 0:
            continue
        P, Q = np.nonzero((rh == h) & (rsgn == 1))
        R, S = np.nonzero((ch == h) & (csgn == 1))
        M = np.zeros((nr, nc))
        M[np.ix_(ridx[P, Q], cidx[R, S])] = dense[P[:, None], Q[:, None], R[None, :], S[None, :]]
        lib.putlst(M, 1, h + 1, lst)


def get_dense_list(lib, dpd, lst, tl, tr):
    """GETLST every irrep of list `lst` into a dense [p,q,r,s] array (absent and
    symmetry-forbidden elements are zero, swapped PACK elements carry sign)."""
    ridx, rsgn, rh = dpd.table(tl)
    cidx, csgn, ch = dpd.table(tr)
    shape = ridx.shape + cidx.shape
    out = np.zeros(shape)
    for h in range(dpd.nirrep):
        nr, nc = lib.list_dims(h + 1, lst)
        if nr == 0 or nc == 0:
            continue
        M = lib.getlst(1, nc, h + 1, lst)
        P, Q = np.nonzero((rh == h) & (rsgn != 0))
        R, S = np.nonzero((ch == h) & (csgn != 0))
        vals = M[np.ix_(ridx[P, Q], cidx[R, S])]
        fr = np.where(rsgn == 2, 1, rsgn).astype(float)
        fc = np.where(csgn == 2, 1, csgn).astype(float)
        sg = fr[P, Q][:, None] * fc[R, S][None, :]
        out[P[:, None], Q[:, None], R[None, :], S[None, :]] = vals * sg
    return out
