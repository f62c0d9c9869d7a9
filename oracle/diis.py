"""DIIS extrapolation as the reference's xvcc performs it -- oracle.

Restates vcc/dodiis0.F:37-243 and libr/dodiis.F:4-87:

* a circular history of ``exporder`` (IFLAGS(12), CC_EXPORDER) iterates; the
  slot written in cycle k is 1 + mod(k-1, exporder) (vcc/dodiis0.F:37-38);
* iterate x_k = the amplitudes that entered the cycle, error e_k = x_new - x_k
  (vcc/dodiis0.F:87-88);
* B(i,j) = <e_i, e_j>, kept across cycles, only the new row/column is
  recomputed (vcc/dodiis0.F:98-129);
* the bordered system [[0, -1], [-1, B]] (lam, c) = (-1, 0) is solved by LU
  with partial pivoting (LAPACK dgesv, libr/dodiis.F:31-46);
* the "largest element of residual vector" is the signed element of e_k of
  largest magnitude, the DIIS residual that of sum c_i e_i; convergence when
  |largest residual| < 10^-CC_CONV (vcc/dodiis0.F:141-176);
* with at least two iterates the new amplitudes are sum_i c_i (x_i + e_i)
  (vcc/dodiis0.F:188-243).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg


def signed_absmax(x):
    """ISAMAX-style: first element of largest magnitude, with its sign."""
    return float(x[int(np.argmax(np.abs(x)))])


class ReferenceDIIS:
    def __init__(self, exporder=5):
        if exporder > 25:
            raise ValueError("at most 25 DIIS iterates (vcc/diislst.F:30 ld_diis)")
        self.n = exporder
        self.R = np.zeros((25, 25))
        self.x = [None] * exporder
        self.e = [None] * exporder

    def step(self, icycle, x_old, x_new):
        """Returns (largest residual, largest DIIS residual, extrapolated
        vector or None when fewer than two iterates exist)."""
        ndimr = min(icycle, self.n)
        idimr = (icycle - 1) % self.n          # 0-based slot
        e = x_new - x_old
        self.x[idimr] = x_old.copy()
        self.e[idimr] = e
        res = signed_absmax(e)
        for i in range(ndimr):
            val = float(np.dot(self.e[i], e))
            self.R[i, idimr] = val
            self.R[idimr, i] = val
        c = self.solve(self.R[:ndimr, :ndimr])
        dvec = np.zeros_like(e)
        for i in range(ndimr):
            dvec += c[i] * self.e[i]
        dres = signed_absmax(dvec)
        if ndimr >= 2:
            ext = dvec.copy()
            for i in range(ndimr):
                ext += c[i] * self.x[i]
            return res, dres, ext
        return res, dres, None

    @staticmethod
    def solve(Bm):
        """libr/dodiis.F: bordered DIIS system, LU with partial pivoting."""
        n = Bm.shape[0]
        A = np.zeros((n + 1, n + 1))
        A[0, 1:] = -1.0
        A[1:, 0] = -1.0
        A[1:, 1:] = Bm
        rhs = np.zeros(n + 1)
        rhs[0] = -1.0
        lu, piv = scipy.linalg.lu_factor(A)
        sol = scipy.linalg.lu_solve((lu, piv), rhs)
        return sol[1:]
