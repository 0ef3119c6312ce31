"""CPU oracle for the Camp-King converger (test infrastructure only).

Only tests/, __graft_entry__.smoke() and the CPU legs of bench.py may import
this module; the product package never does.  It is the checker, not the
thing measured or shipped.

What it restates (closed-shell RHF, the alpha call of iter):
  * ``interp`` (matrix/interp.F90:16-346), R. N. Camp and H. F. King,
    J. Chem. Phys. 75, 268 (1981): the corresponding-orbital analysis of the
    new and the old vectors, the energy derivative along the rotation, the
    cubic-spline search for the rotation angle and the rotated vectors;
  * ``spline`` (interp.F90:349-484);
  * ``schmit`` / ``schmib`` (matrix/schmit.F90, matrix/schmib.F90): modified
    Gram-Schmidt over the columns in order / in reverse order, with the
    reference's re-orthogonalisation passes and unit-vector fallback;
  * ``rsp`` (matrix/rsp.F90): eigenvectors_LAPACK for n > 1.

As in this version of the reference, ``emin`` is set to 0 once per
calculation and never updated (spline's minimum stays local to spline), so
the interpolation step is taken only while eold - e <= 0.9 eold, i.e. for a
positive heat of formation; for a negative one interp analyses the vectors
every iteration and never rotates them.
"""
from __future__ import annotations

import math

import numpy as np

from oracle.scf_oracle import eigenvectors_lapack, unpack


def schmit(u: np.ndarray, n: int) -> None:
    """schmit.F90:16-62 on the n x n block u[:n, :n] (in place): columns in
    order, each normalised, then projected on the earlier ones one at a time
    (modified Gram-Schmidt) until its remaining norm^2 is at least 0.01 (at
    most three passes); a column that vanishes is replaced by the next unit
    vector e_ii (only that element is set) and projected again."""
    small = 0.01
    ii = 0
    for k in range(n):
        col = u[:n, k]
        dot = float(col @ col)
        if abs(dot) < 1.0e-20:
            state = 100
        else:
            col *= 1.0 / math.sqrt(dot)
            state = 30
        npass = 0
        while True:
            if state == 100:
                ii += 1
                if ii <= n:
                    u[ii - 1, k] = 1.0
                state = 30
            if state == 30:
                if k == 0:
                    break
                npass = 0
                state = 40
            # state 40
            npass += 1
            for j in range(k):
                d = float(u[:n, j] @ col)
                col -= d * u[:n, j]
            dot = float(col @ col)
            if abs(dot) < 1.0e-20 or (dot < small and npass > 2):
                state = 100
                continue
            col *= 1.0 / math.sqrt(dot)
            if dot < small:
                state = 40
                continue
            break


def schmib(u: np.ndarray, n: int) -> None:
    """schmib.F90:16-63: schmit over the columns n-1, n-2, ..., 0."""
    schmit(u[:n, :n][:, ::-1], n)


def rsp(hpacked: np.ndarray, n: int):
    """rsp.F90:16-33: eigenvalues (ascending) and eigenvectors (columns) of a
    packed symmetric matrix; eigenvectors_LAPACK (which perturbs the packed
    input in place) for n > 1."""
    if n == 1:
        return np.array([hpacked[0]]), np.ones((1, 1))
    v, w = eigenvectors_lapack(hpacked, n)
    return w, v


def spline(x, f, df, xhigh: float, xlow: float, npnts: int) -> float:
    """interp.F90:349-484.  x, f, df: 1-based lists (index 0 unused) that the
    call reorders (the newest point, at npnts, is inserted in x order);
    returns xmin, the abscissa of the lowest point or cubic minimum found
    between xlow and xhigh."""
    close, big, huge, ustep, dstep = 1.0e-8, 500.0, 1.0e10, 1.0, 2.0
    xmin, fmin, dfmin = x[npnts], f[npnts], df[npnts]
    n1 = npnts - 1
    j2 = min(1, n1)
    k = n1
    while k >= j2:  # the DO loop leaves k = j2 - 1 when it runs out
        if x[k] < xmin:
            break
        x[k + 1], f[k + 1], df[k + 1] = x[k], f[k], df[k]
        k -= 1
    x[k + 1], f[k + 1], df[k + 1] = xmin, fmin, dfmin
    step = dstep if df[1] > 0.0 else ustep
    xstart = max(x[1] - step * (x[2] - x[1]), xlow)
    step = ustep if df[npnts] > 0.0 else dstep
    xstop = min(x[npnts] + step * (x[npnts] - x[n1]), xhigh)
    for k in range(1, n1 + 1):
        skip1 = k != 1
        skip2 = k != n1
        if f[k] < fmin:
            xmin, fmin, dfmin = x[k], f[k], df[k]
        dx = x[k + 1] - x[k]
        if dx <= close:
            continue
        x1 = xstart - x[1] if k == 1 else 0.0
        x2 = xstop - x[n1] if k == n1 else dx
        dum = (f[k + 1] - f[k]) / dx
        a = (df[k] + df[k + 1] - dum - dum) / (dx * dx)
        b = (dum + dum + dum - df[k] - df[k] - df[k + 1]) / dx
        c = df[k]
        bb = b * b
        ac3 = (a + a + a) * c
        xk = None                       # None: no interior cubic minimum (label 90)
        if not bb < ac3:
            if b <= 0.0:
                if not abs(b) > huge * abs(a):
                    xk = (-b + math.sqrt(bb - ac3)) / (a + a + a)
            elif bb > big * abs(ac3):   # label 60: series for a small ac3/bb
                r = ac3 / bb
                xk = -(((0.039063 * r + 0.0625) * r + 0.125) * r + 0.5) * c / b
            else:
                xk = (-b + math.sqrt(bb - ac3)) / (a + a + a)
            if xk is not None and (xk < x1 or xk > x2):
                xk = None
        while True:
            if xk is not None:          # label 80
                fm = ((a * xk + b) * xk + c) * xk + f[k]
                if fm <= fmin:
                    xmin = xk + x[k]
                    fmin = fm
                    dfmin = ((a + a + a) * xk + b + b) * xk + c
            if not skip1:               # label 90: the interval's left end
                skip1 = True
                xk = x1
                continue
            if not skip2:               # label 100: its right end
                skip2 = True
                xk = x2
                continue
            break
    return xmin


class CampKing:
    """interp's saved state (the SAVE variables and iter's vec_ai, fock_ai,
    p_ai, h_ai, theta and eold_alpha) for one calculation."""

    def __init__(self, n: int):
        self.n = n
        self.vec = np.zeros((n, n), order="F")
        self.fock = np.zeros((n, n), order="F")
        self.p = np.zeros((n, n), order="F")
        self.theta = np.zeros(n)
        self.x = [0.0] * 13
        self.f = [0.0] * 13
        self.df = [0.0] * 13
        self.xold = 0.0
        self.xnow = 0.0
        self.xlow = 0.0
        self.xhigh = 0.0
        self.npnts = 0
        self.ipoint = 0
        self.emin = 0.0
        self.eold_ref = 0.0
        self.rotations = 0     # interpolation steps taken (mode 3 returns)

    def interp(self, np_: int, nq: int, mode: int, e: float, fp: np.ndarray, cp: np.ndarray) -> int:
        """interp.F90:16-346 for np_ filled and nq empty levels; e: the energy
        (escf / 23.06...), fp: packed Fock matrix, cp: the vectors (n x n,
        replaced by the rotated ones on a mode 3 return).  Returns the new
        mode: 2 (analyse the next vectors), 3 (cp holds the interpolated
        vectors: build their density without diagonalising)."""
        n = self.n
        m = min(np_, nq)
        F = unpack(fp, n)
        PI, VEC, FK, theta = self.p, self.vec, self.fock, self.theta
        if mode != 2:
            # :86-109  F C_v and the occupied-virtual block C_o^T F C_v
            PI[:, :nq] = F @ cp[:, np_:np_ + nq]
            FK[:np_, :nq] = cp[:, :np_].T @ PI[:, :nq]
            if mode != 3:                       # :110-118 the current point becomes the old one
                VEC[:, :] = cp
                self.eold_ref = e
                self.xold = 1.0
                return 2
            self.npnts += 1                     # :125-127 an interpolated point
            self.ipoint = self.npnts
        else:
            # :135-142  overlaps of the new vectors with the old ones
            # (the block rows >= np, columns < np is not formed)
            PI[:np_, :] = cp[:, :np_].T @ VEC
            PI[np_:, np_:] = cp[:, np_:].T @ VEC[:, np_:]
            sov = PI[:np_, np_:]
            # :147-155  H = S_ov S_ov^T and its eigenvectors
            hp = _pack_lower_rows(sov @ sov.T)
            w, v = rsp(hp, np_)
            theta[:np_] = w
            VEC[:np_, :np_] = v
            # :156-169  descending order
            theta[:np_] = theta[:np_][::-1].copy()
            VEC[:np_, :np_] = VEC[:np_, :np_][:, ::-1].copy()
            # :170-174  rotation angles
            for i in range(m):
                theta[i] = math.asin(math.sqrt(min(max(theta[i], 0.0), 1.0)))
            # :180-186  W_q = S_ov^T V_p (first m columns), orthonormalised
            VEC[:nq, np_:np_ + m] = sov.T @ VEC[:np_, :m]
            schmit(VEC[:, np_:], nq)
            # :191-208  U_p = S_oo^T V_p, orthonormalised in reverse order
            PI[:np_, :np_] = PI[:np_, :np_].T.copy()
            PI[:np_, :np_] = PI[:np_, :np_] @ VEC[:np_, :np_]
            schmib(PI, np_)
            # :212-219  U_q = S_vv W_q, orthonormalised in reverse order
            svv = PI[np_:np_ + nq, np_:np_ + nq].copy()
            PI[:nq, np_:np_ + nq] = svv @ VEC[:nq, np_:np_ + nq]
            schmib(PI[:, np_:], nq)
            # :223-237  dE/dx at the old point
            a = PI[:np_, :m] * theta[:m]
            d = a @ VEC[:nq, np_:np_ + m].T
            dedx = float(np.sum(d * FK[:np_, :nq]))
            deold = -4.0 * dedx
            self.x[2], self.f[2], self.df[2] = self.xold, self.eold_ref, deold
            # :241-254  the corresponding current orbitals
            PI[:np_, :np_] = VEC[:np_, :np_]
            vnew = np.empty((n, n), order="F")
            vnew[:, :np_] = cp[:, :np_] @ PI[:np_, :np_]
            vnew[:, np_:] = cp[:, np_:np_ + nq] @ PI[:nq, np_:np_ + nq]
            VEC[:, :] = vnew
            # :260-294  F in the corresponding representation
            PI[:, :nq] = F @ VEC[:, np_:np_ + nq]
            FK[:np_, :nq] = VEC[:, :np_].T @ PI[:, :nq]
            self.npnts = 2
            self.ipoint = 1
            self.xnow = 0.0
            with np.errstate(divide="ignore"):
                self.xhigh = float(np.float64(math.pi) / (2.0 * np.float64(theta[0])))
            self.xlow = -0.5 * self.xhigh
        # :301-312  the current point and the spline
        dedx = float(np.sum(theta[:m] * np.diagonal(FK)[:m]))
        denow = -4.0 * dedx
        enow = e
        ip = self.ipoint
        self.x[ip], self.f[ip], self.df[ip] = self.xnow, enow, denow
        xmin = spline(self.x, self.f, self.df, self.xhigh, self.xlow, self.npnts)
        if self.eold_ref - enow <= 0.9 * (self.eold_ref - self.emin) and ip <= 10:
            # :313-327  rotate to the interpolated angle
            self.xnow = xmin
            cp[:, :] = VEC
            for k in range(m):
                ck = math.cos(self.xnow * theta[k])
                sk = math.sin(self.xnow * theta[k])
                cp[:, k] = ck * VEC[:, k] - sk * VEC[:, np_ + k]
                cp[:, np_ + k] = sk * VEC[:, k] + ck * VEC[:, np_ + k]
            self.rotations += 1
            return 3
        if mode != 2:                           # :333-337
            VEC[:, :] = cp
            mode = 2
        self.eold_ref = enow
        return mode


def _pack_lower_rows(a: np.ndarray) -> np.ndarray:
    """Lower triangle by rows (MOPAC's packed layout): h(ij), j <= i."""
    r, c = np.tril_indices(a.shape[0])
    return np.ascontiguousarray(a[r, c])
