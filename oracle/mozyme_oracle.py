"""CPU oracle for the MOZYME sparse-block kernels (test infrastructure only).

Only tests/ and the CPU legs of bench.py may import this module.  It binds the
C restatements in mopac_oracle.c:
  * orc_mz_layout   -- fillij (MOZYME/fillij.F90:20-230), first call, id = 0;
  * orc_mz_density  -- density_for_MOZYME (MOZYME/density_for_MOZYME.F90:16-342);
  * orc_mz_helecz   -- helecz (MOZYME/helecz.F90:16-52);
  * orc_mz_cnvgz    -- cnvgz (MOZYME/cnvgz.F90:16-85).
"""
from __future__ import annotations

import ctypes

import numpy as np

from oracle import scf_oracle as so

_bound = False


def _lib():
    global _bound
    L = so.lib()
    if not _bound:
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
        i64p = np.ctypeslib.ndpointer(np.int64, flags="C")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
        L.orc_mz_layout.argtypes = [ctypes.c_int, i32p, f64p, ctypes.c_double, ctypes.c_double, i64p]
        L.orc_mz_layout.restype = ctypes.c_longlong
        L.orc_mz_density.argtypes = [ctypes.c_int, i32p, i64p, ctypes.c_int, i32p, i32p, i32p, i32p, f64p,
                                     ctypes.c_int, ctypes.c_longlong, f64p, f64p]
        L.orc_mz_helecz.argtypes = [ctypes.c_int, i32p, i64p, f64p, f64p, f64p]
        L.orc_mz_helecz.restype = ctypes.c_double
        L.orc_mz_cnvgz.argtypes = [ctypes.c_int, ctypes.c_longlong, f64p, f64p, f64p, f64p, f64p, ctypes.c_int,
                                   i64p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        _bound = True
    return L


def cutoffs(numat: int, cutofp: float | None = None):
    """cutof1, cutof2 (squared) as fillij sets them (MOZYME/fillij.F90:59-80)."""
    c1, c2 = 10.0 ** 2, 9.9 ** 2
    if cutofp is not None and cutofp < 100.0:
        c1, c2 = cutofp ** 2 + 1e-4, cutofp ** 2
    if numat < 30:
        c1, c2 = 1.0e6 + 10, 1.0e6
    return c1, c2


def layout(iorbs, coord, cutof1: float, cutof2: float):
    iorbs = np.ascontiguousarray(iorbs, np.int32)
    coord = np.ascontiguousarray(coord, np.float64).reshape(-1)
    n = iorbs.size
    nijbo = np.zeros(n * n, np.int64)
    mpack = _lib().orc_mz_layout(n, iorbs, coord, cutof1, cutof2, nijbo)
    return int(mpack), nijbo.reshape(n, n)


def idiag(iorbs, nijbo) -> np.ndarray:
    """iter_for_MOZYME.F90:183-190 (1-based positions)."""
    out = []
    for i, io in enumerate(iorbs):
        j = int(nijbo[i, i])
        for k in range(1, int(io) + 1):
            j += k
            out.append(j)
    return np.array(out, np.int64)


def density(iorbs, nijbo, lmos, mode: int, mpack: int, partp=None) -> np.ndarray:
    ncf, nncf, icocc, ncocc, cocc = lmos
    p = np.zeros(mpack)
    pp = np.zeros(mpack) if partp is None else np.ascontiguousarray(partp, np.float64)
    _lib().orc_mz_density(len(iorbs), np.ascontiguousarray(iorbs, np.int32), np.ascontiguousarray(nijbo.ravel()),
                          len(ncf), ncf, nncf, icocc, ncocc, cocc, mode, mpack, pp, p)
    return p


def helecz(iorbs, nijbo, p, h, f) -> float:
    return _lib().orc_mz_helecz(len(iorbs), np.ascontiguousarray(iorbs, np.int32),
                                np.ascontiguousarray(nijbo.ravel()), p, h, f)


def cnvgz(pnew, p, p1, p2, p3, niter: int, idg, use3: bool = True) -> float:
    pm = ctypes.c_double()
    _lib().orc_mz_cnvgz(p1.size, pnew.size, pnew, p, p1, p2, p3, niter, idg, int(use3), ctypes.byref(pm))
    return pm.value


def dense_to_blocks(a: np.ndarray, iorbs, nijbo, mpack: int) -> np.ndarray:
    """Gather a full symmetric matrix into the pair-block storage."""
    first = np.concatenate([[0], np.cumsum(iorbs)[:-1]])
    out = np.zeros(mpack)
    n = len(iorbs)
    for i in range(n):
        for j in range(i + 1):
            off = int(nijbo[i, j])
            if off < 0:
                continue
            bi = a[first[i]:first[i] + iorbs[i], first[j]:first[j] + iorbs[j]]
            if i == j:
                r, c = np.tril_indices(iorbs[i])
                vals = bi[r, c]
            else:
                vals = bi.ravel()
            out[off:off + vals.size] = vals
    return out


def dense_w_offsets(iorbs) -> np.ndarray:
    """Offsets of the dense W blocks (hcore's order): pair (i, j), j < i, and
    the one-centre block (i, i)."""
    n = len(iorbs)
    off = np.zeros((n, n), np.int64)
    kk = 0
    for i in range(n):
        for j in range(i):
            off[i, j] = kk
            a, b = iorbs[i] >= 3, iorbs[j] >= 3
            kk += 100 if (a and b) else (10 if (a or b) else 1)
        off[i, i] = kk
        il = iorbs[i] * (iorbs[i] + 1) // 2
        kk += il * il
    return off


def w_stored(iorbs, nijbo, w_dense) -> np.ndarray:
    """The dense W with the blocks of pairs outside cutof2 left out: the
    integrals fock2z uses, in the layout's entry order."""
    off = dense_w_offsets(iorbs)
    out = []
    n = len(iorbs)
    for i in range(n):
        for j in range(i):
            if nijbo[i, j] >= 0:
                a, b = iorbs[i] >= 3, iorbs[j] >= 3
                sz = 100 if (a and b) else (10 if (a or b) else 1)
                out.append(w_dense[off[i, j]:off[i, j] + sz])
        il = iorbs[i] * (iorbs[i] + 1) // 2
        out.append(w_dense[off[i, i]:off[i, i] + il * il])
    return np.ascontiguousarray(np.concatenate(out))


def fock(nat, coord, iorbs, nijbo, w_dense, ptot, h):
    """fz2n mode 0: F from H (both in the pair-block storage)."""
    L = _lib()
    if not hasattr(L, "_mz_fock_bound"):
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
        i64p = np.ctypeslib.ndpointer(np.int64, flags="C")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
        L.orc_mz_fock.argtypes = [ctypes.c_int, i32p, f64p, i32p, i64p, f64p, f64p, f64p, f64p]
        L._mz_fock_bound = True
    f = np.ascontiguousarray(h, np.float64).copy()
    qe = np.zeros(len(iorbs))
    L.orc_mz_fock(len(iorbs), np.ascontiguousarray(nat, np.int32), np.ascontiguousarray(coord, np.float64).ravel(),
                  np.ascontiguousarray(iorbs, np.int32), np.ascontiguousarray(nijbo.ravel()),
                  np.ascontiguousarray(w_dense, np.float64), np.ascontiguousarray(ptot, np.float64), f, qe)
    return f


def diagg1(iorbs, nijbo, fao, p, occ, vir, idiagg, state, nfmo, ifmo, fmo, cap):
    """diagg1 (MOZYME/diagg1.F90:16-503), lijbo path.  state = [fref, safety,
    oldlim, tiny] (updated in place); nfmo, ifmo (2 x cap), fmo (cap) carry
    the list between calls.  Returns (nij, eigv, eigs or None, sumt)."""
    L = _lib()
    if not hasattr(L, "_mz_diagg1_bound"):
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
        i64p = np.ctypeslib.ndpointer(np.int64, flags="C")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
        L.orc_mz_diagg1.argtypes = ([ctypes.c_int, i32p, i32p, ctypes.c_int, i64p, f64p, f64p, ctypes.c_int]
                                    + [i32p] * 4 + [f64p, ctypes.c_int] + [i32p] * 4
                                    + [f64p, ctypes.c_int, f64p, i32p, i32p, f64p, ctypes.POINTER(ctypes.c_longlong),
                                       f64p, f64p, ctypes.POINTER(ctypes.c_int)])
        L.orc_mz_diagg1.restype = ctypes.c_double
        L._mz_diagg1_bound = True
    iorbs = np.ascontiguousarray(iorbs, np.int32)
    first = np.ascontiguousarray(np.concatenate([[0], np.cumsum(iorbs)[:-1]]), np.int32)
    ncf, nncf, icocc, ncocc, cocc = occ
    nce, nnce, icvir, ncvir, cvir = vir
    eigv = np.zeros(len(nce))
    eigs = np.zeros(len(ncf))
    nij = ctypes.c_longlong(cap)
    done = ctypes.c_int(0)
    sumt = L.orc_mz_diagg1(len(iorbs), iorbs, first, int(iorbs.sum()), np.ascontiguousarray(nijbo.ravel()),
                           np.ascontiguousarray(fao), np.ascontiguousarray(p), len(ncf), ncf, nncf, icocc, ncocc,
                           cocc, len(nce), nce, nnce, icvir, ncvir, cvir, idiagg, state, nfmo, ifmo, fmo,
                           ctypes.byref(nij), eigv, eigs, ctypes.byref(done))
    return nij.value, eigv, (eigs if done.value else None), sumt


def diagg2(iorbs, occ, vir, ifmo, fmo, nij, eigs, eigv, idiagg, ctl, nrejct):
    """diagg2 (MOZYME/diagg2.F90:16-359).  occ/vir tuples of numpy arrays are
    modified in place (ncf, icocc, cocc / nce, icvir, cvir); nrejct (int32[2])
    updated.  Returns (sumb, nrej)."""
    L = _lib()
    if not hasattr(L, "_mz_diagg2_bound"):
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
        L.orc_mz_diagg2.argtypes = ([ctypes.c_int, i32p, ctypes.c_int, ctypes.c_int, i32p, i32p, i32p, i32p, f64p,
                                     ctypes.c_longlong, ctypes.c_longlong, ctypes.c_int, i32p, i32p, i32p, i32p, f64p,
                                     ctypes.c_longlong, ctypes.c_longlong, i32p, f64p, ctypes.c_longlong, f64p, f64p,
                                     ctypes.c_int, f64p, i32p, ctypes.POINTER(ctypes.c_longlong)])
        L.orc_mz_diagg2.restype = ctypes.c_double
        L._mz_diagg2_bound = True
    iorbs = np.ascontiguousarray(iorbs, np.int32)
    ncf, nncf, icocc, ncocc, cocc = occ
    nce, nnce, icvir, ncvir, cvir = vir
    nrej = ctypes.c_longlong(0)
    sumb = L.orc_mz_diagg2(len(iorbs), iorbs, int(iorbs.sum()), len(ncf), ncf, nncf, icocc, ncocc, cocc,
                           icocc.size, cocc.size, len(nce), nce, nnce, icvir, ncvir, cvir, icvir.size, cvir.size,
                           np.ascontiguousarray(ifmo, np.int32), np.ascontiguousarray(fmo, np.float64), int(nij),
                           np.ascontiguousarray(eigs), np.ascontiguousarray(eigv), int(idiagg),
                           np.ascontiguousarray(ctl, np.float64), nrejct, ctypes.byref(nrej))
    return sumb, nrej.value
