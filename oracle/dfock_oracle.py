"""CPU oracle for dfock2, the two-centre Fock-matrix derivative of one atom
(test infrastructure only).

Only tests/, __graft_entry__.smoke() and the CPU legs of bench.py may import
this module; the product package never does.  It is the checker, not the
thing measured or shipped.

Restates forces/dfock2.F90:16-279 (the itype = 3 path, the only one the
routine reaches) for an sp basis: for every atom jj != nati in ascending
order, the pair's block of the derivative integrals w (100, 10 or 1 values
for heavy-heavy, heavy-light or light-light pairs, in partner order) adds
jab's Coulomb terms (integrals/jab.F90) and kab's exchange terms
(integrals/kab.F90), or the light-atom forms of both, to f.  Python floats
round like the reference's double precision arithmetic without fused
multiply-adds, and every sum runs in the reference's term order, so the
result is the reference's bit for bit.

Arrays: f, ptot, p packed lower triangles by rows (MOPAC's layout, 0-based
here: element (i, j), i >= j, at i (i + 1) / 2 + j); nfirst, nlast 1-based
orbital ranges per atom as in the reference; nati 1-based.
"""
from __future__ import annotations

import numpy as np


def _pair1(a: int, b: int) -> int:
    """1-based index of the orbital pair (a, b), 1 <= a, b <= 4."""
    hi, lo = max(a, b), min(a, b)
    return hi * (hi - 1) // 2 + lo


# jab's density gather / kab's term order / dfock2's jindex(1..16):
# term m (0-based) uses pair (m // 4 + 1, m % 4 + 1)
PIDX = [_pair1(m // 4 + 1, m % 4 + 1) for m in range(16)]


def _ix(i: int, j: int) -> int:
    """0-based packed index of 1-based orbitals i, j."""
    hi, lo = max(i, j), min(i, j)
    return hi * (hi - 1) // 2 + lo - 1


def partner_sizes(nfirst, nlast, nati: int):
    """Per-partner block sizes of w (dfock2.F90:106, :155, :204, :216) and
    their offsets kk, in partner order; nati 1-based."""
    numat = len(nfirst)
    heavy_i = nlast[nati - 1] - nfirst[nati - 1] >= 3
    off, kk = {}, 0
    for jj in range(1, numat + 1):
        if jj == nati:
            continue
        heavy_j = nlast[jj - 1] - nfirst[jj - 1] >= 3
        off[jj] = kk
        kk += 100 if (heavy_i and heavy_j) else (10 if (heavy_i or heavy_j) else 1)
    return off, kk


def dfock2(f: np.ndarray, ptot: np.ndarray, p: np.ndarray, w: np.ndarray, nfirst, nlast, nati: int) -> None:
    """forces/dfock2.F90:16-279 (in place on f)."""
    numat = len(nfirst)
    ia, ib = nfirst[nati - 1], nlast[nati - 1]
    kk = 0
    for jj in range(1, numat + 1):
        if jj == nati:
            continue
        ja, jb = nfirst[jj - 1], nlast[jj - 1]
        if ib - ia >= 6 or jb - ja >= 6:
            raise ValueError("d orbitals are outside this restatement")
        if ib - ia >= 3 and jb - ja >= 3:
            # jab (:79-82) with pja, pjb the two diagonal blocks, 4 x 4
            pja = [ptot[_ix(ia + m // 4, ia + m % 4)] for m in range(16)]
            pjb = [ptot[_ix(ja + m // 4, ja + m % 4)] for m in range(16)]
            W = lambda r, c: w[kk + 10 * (r - 1) + c - 1]   # noqa: E731 (1-based row, column)
            suma, sumb = [], []
            for r in range(1, 11):
                s = pja[0] * W(PIDX[0], r)
                for m in range(1, 16):
                    s = s + pja[m] * W(PIDX[m], r)
                suma.append(s)
                s = pjb[0] * W(r, PIDX[0])
                for m in range(1, 16):
                    s = s + pjb[m] * W(r, PIDX[m])
                sumb.append(s)
            i = 0
            for i5 in range(1, 5):
                for i6 in range(1, i5 + 1):
                    f[_ix(ia + i5 - 1, ia + i6 - 1)] += sumb[i]
                    f[_ix(ja + i5 - 1, ja + i6 - 1)] += suma[i]
                    i += 1
            # kab (:83-104) with pk(4 (i - ia) + (j - ja) + 1) = P(i, j)
            pk = [p[_ix(ia + m // 4, ja + m % 4)] for m in range(16)]
            sums = []
            for a in range(4):
                for b in range(4):
                    s = None
                    for k in range(16):
                        t = pk[k] * W(_pair1(a + 1, k // 4 + 1), _pair1(b + 1, k % 4 + 1))
                        s = t if s is None else s + t
                    sums.append(s)
            if ia > ja:
                m = 0
                for j1 in range(ia, ia + 4):
                    for j in range(4):
                        f[_ix(j1, ja + j)] -= sums[m]
                        m += 1
            else:
                m = 0
                for j1 in range(ia, ia + 4):
                    for j2 in range(ja, ja + 4):
                        f[_ix(j2, j1)] -= sums[m]
                        m += 1
            kk += 100
        elif ib - ia >= 3 or jb - ja >= 3:
            # :106-203 one heavy (h) and one light (l) atom; the heavy atom's
            # block takes ptot(ll) w, the light atom's diagonal the two sums
            h0, l0 = (ia, ja) if ib - ia >= 3 else (ja, ia)
            ll = _ix(l0, l0)
            sumdia = 0.0
            sumoff = 0.0
            k = 0
            for i in range(4):
                for j in range(i):
                    j1 = _ix(h0 + i, h0 + j)
                    f[j1] += ptot[ll] * w[kk + k]
                    sumoff = sumoff + ptot[j1] * w[kk + k]
                    k += 1
                j1 = _ix(h0 + i, h0 + i)
                f[j1] += ptot[ll] * w[kk + k]
                sumdia = sumdia + ptot[j1] * w[kk + k]
                k += 1
            f[ll] = f[ll] + sumoff * 2.0 + sumdia
            # exchange: f(h + i, l) -= sum_j p(h + j, l) w(jindex(4 i + j + 1))
            for i in range(4):
                s = 0.0
                for j in range(4):
                    s = s + p[_ix(h0 + j, l0)] * w[kk + PIDX[4 * i + j] - 1]
                f[_ix(h0 + i, l0)] -= s
            kk += 10
        else:
            # :204-215 two light atoms
            i1, j1 = _ix(ia, ia), _ix(ja, ja)
            f[i1] += ptot[j1] * w[kk]
            f[j1] += ptot[i1] * w[kk]
            ij = _ix(ia, ja)
            f[ij] -= p[ij] * w[kk]
            kk += 1
