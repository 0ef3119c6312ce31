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


# ------------------------------------------------------------ the SCF loop
# The MOZYME SCF (iter_for_MOZYME) on the oracle's kernels, with the routines
# its loop calls between them: check, eimp, hbonds/addhb, isitsc, and a
# starting-LMO builder for water that stands in for makvec.

def check_lmos(lmos, iorbs) -> float:
    """check (MOZYME/check.F90:1-60): renormalise every LMO over its atoms;
    returns the summed |1 - norm^2| (the reference stops above 0.1)."""
    ncf, nncf, icocc, ncocc, cocc = lmos
    err = 0.0
    for i in range(len(ncf)):
        n = int(sum(iorbs[icocc[nncf[i] + j] - 1] for j in range(ncf[i])))
        ssum = 0.0
        for m in range(ncocc[i], ncocc[i] + n):   # the reference's order
            ssum += float(cocc[m]) * float(cocc[m])
        err += abs(1.0 - ssum)
        cocc[ncocc[i]:ncocc[i] + n] *= 1.0 / np.sqrt(ssum)
    return err


def tidy(lmos, iorbs, thresh: float = 1.0e-13) -> None:
    """The compression step of tidy (MOZYME/tidy.F90:66-107): every LMO drops
    the atoms whose squared coefficients sum to thresh or less, keeping the
    order of the rest, in place within its own storage.  (The reference then
    repacks all LMOs and spreads the free space evenly, :133-213; here every
    LMO keeps its own fixed space, so only the counts and contents change.)"""
    ncf, nncf, icocc, ncocc, cocc = lmos
    for i in range(len(ncf)):
        mm = ncocc[i]
        mn = ncocc[i]
        kept = 0
        for j1 in range(ncf[i]):
            a = icocc[nncf[i] + j1]
            no = int(iorbs[a - 1])
            ssum = 0.0
            for k in range(no):
                ssum += float(cocc[mm + k]) ** 2
            if ssum > thresh:
                cocc[mn:mn + no] = cocc[mm:mm + no].copy()
                icocc[nncf[i] + kept] = a
                mn += no
                kept += 1
            mm += no
        ncf[i] = kept


def eimp(iorbs, nijbo, p, f) -> None:
    """eimp (MOZYME/eimp.F90): the first element of every stored
    off-diagonal block of p becomes that block's sum of squared F elements,
    the pair weight diagg1 reads (the next density build overwrites it)."""
    for i in range(len(iorbs)):
        for j in range(i):
            k = int(nijbo[i, j])
            if k >= 0:
                acc = 0.0
                for q in range(k, k + int(iorbs[i] * iorbs[j])):
                    acc += float(f[q]) * float(f[q])
                p[k] = acc


HB_LIMITS = (1.0, 0.1, 0.01, 0.001)   # addhb.F90: hblims


def hbonds(iorbs, nijbo, fao, p, occ, vir, cutoff: float, cap: int):
    """hbonds (MOZYME/hbonds.F90): for every stored atom pair (i > j) with no
    density yet (sum P^2 < 1e-10) but a Fock block above cutoff, every
    virtual LMO whose first or second atom is i or j paired with every
    occupied LMO of that kind, with the nominal element 0.1, in the
    reference's loop order.  Returns (nij, ifmo, fmo) in diagg1's layout."""
    ncf, nncf, icocc = occ[0], occ[1], occ[2]
    nce, nnce, icvir = vir[0], vir[1], vir[2]
    ifmo = np.zeros(2 * cap, np.int32)
    fmo = np.zeros(cap)
    nij = 0
    for i in range(len(iorbs)):
        for j in range(i):
            k = int(nijbo[i, j])
            if k < 0:
                continue
            sumf = sump = 0.0
            for q in range(k, k + int(iorbs[i] * iorbs[j])):
                sumf += float(fao[q]) * float(fao[q])
                sump += float(p[q]) * float(p[q])
            if not (sump < 1.0e-10 and sumf > cutoff):
                continue
            used = []
            for q in range(len(ncf)):
                kk = min(int(ncf[q]) - 1, 1)
                l0 = int(nncf[q])
                if icocc[l0] - 1 in (i, j) or icocc[l0 + kk] - 1 in (i, j):
                    used.append(q)
            for q in range(len(nce)):
                kk = min(int(nce[q]) - 1, 1)
                l0 = int(nnce[q])
                if icvir[l0] - 1 in (i, j) or icvir[l0 + kk] - 1 in (i, j):
                    for u in used:
                        if nij >= cap:
                            raise RuntimeError("hbonds: list capacity exceeded")
                        fmo[nij] = 0.1
                        ifmo[2 * nij] = q + 1
                        ifmo[2 * nij + 1] = u + 1
                        nij += 1
    return nij, ifmo, fmo


def _pipek_mezey(C: np.ndarray, atom_of: np.ndarray, natoms: int, sweeps: int = 100) -> np.ndarray:
    """Pipek-Mezey localisation (Jacobi sweeps) of the columns of C in an
    orthonormal AO basis (NDDO): maximises sum over MOs and atoms of the
    squared atomic populations."""
    C = C.copy()
    n = C.shape[1]
    masks = [atom_of == a for a in range(natoms)]
    for _ in range(sweeps):
        biggest = 0.0
        for i in range(n):
            for j in range(i + 1, n):
                A = B = 0.0
                for m in masks:
                    qii = float(np.sum(C[m, i] ** 2))
                    qjj = float(np.sum(C[m, j] ** 2))
                    qij = float(np.sum(C[m, i] * C[m, j]))
                    A += qij * qij - 0.25 * (qii - qjj) ** 2
                    B += qij * (qii - qjj)
                if A * A + B * B < 1.0e-24:
                    continue
                g = 0.25 * np.arccos(-A / np.hypot(A, B)) * (1.0 if B >= 0.0 else -1.0)
                c, s = np.cos(g), np.sin(g)
                ci, cj = C[:, i].copy(), C[:, j].copy()
                C[:, i] = c * ci + s * cj
                C[:, j] = -s * ci + c * cj
                biggest = max(biggest, abs(g))
        if biggest < 1.0e-10:
            break
    return C


def water_lewis_lmos(nat, xyz, pad_atoms: int = 0):
    """Starting LMOs for (H2O)_n in MOZYME_C's arrays, standing in for makvec
    (its Lewis-structure builder is out of scope): per molecule, the isolated
    molecule's occupied and virtual canonical MOs, Pipek-Mezey localised
    (two O-H bonds + two lone pairs; two O-H antibonds), each LMO's atoms
    listed by falling weight so its first two atoms are its bond's atoms, as
    hbonds expects.  pad_atoms spare atom slots follow every LMO (room for
    diagg2 to grow it).  Returns (iorbs, occ, vir)."""
    nat = np.asarray(nat)
    xyz = np.asarray(xyz, float).reshape(-1, 3)
    iorbs = np.where(nat == 1, 1, 4).astype(np.int32)
    occ = ([], [], [], [], [])
    vir = ([], [], [], [], [])
    atom_of = np.array([0, 0, 0, 0, 1, 2])
    for m in range(len(nat) // 3):
        a = [3 * m, 3 * m + 1, 3 * m + 2]
        if not (nat[a[0]] == 8 and nat[a[1]] == 1 and nat[a[2]] == 1):
            raise ValueError("water_lewis_lmos: atoms must come as O, H, H")
        r1 = so.iter_scf(so.make_system(nat[a], xyz[a]), scfcrt=1.0e-8)
        for C, dst in ((_pipek_mezey(r1.c[:, :4], atom_of, 3), occ), (_pipek_mezey(r1.c[:, 4:6], atom_of, 3), vir)):
            for col in range(C.shape[1]):
                v = C[:, col]
                w = np.array([np.sum(v[:4] ** 2), v[4] ** 2, v[5] ** 2])
                ncf, nncf, icocc, ncocc, cocc = dst
                nncf.append(len(icocc))
                ncocc.append(len(cocc))
                ncf.append(3)
                for o in np.argsort(-w, kind="stable"):
                    icocc.append(a[o] + 1)
                    cocc.extend(v[:4].tolist() if o == 0 else [float(v[3 + o])])
                icocc.extend([0] * pad_atoms)
                cocc.extend([0.0] * (4 * pad_atoms))
    cast = lambda t: (np.array(t[0], np.int32), np.array(t[1], np.int32), np.array(t[2], np.int32),
                      np.array(t[3], np.int32), np.array(t[4], np.float64))
    return iorbs, cast(occ), cast(vir)


def iter_for_mozyme(s, occ, vir, cutof1: float, cutof2: float, scfcrt: float = 1.0e-2, itrmax: int = 2000,
                    trace: bool = False):
    """The MOZYME SCF loop (MOZYME/iter_for_MOZYME.F90:218-630) for a whole
    closed-shell system (numred = numat: no partial SCF, no setupk):
    density, Fock and energy of the starting LMOs (:439-473); then per
    iteration check (:482-484), eimp (:495), diagg = diagg1 + diagg2 +
    density (diagg.F90), addhb every third iteration while nhb < 4
    (:529-538, addhb.F90, hbonds.F90), cnvgz while the three-point
    extrapolation is on (:549), buildf and helecz (:558-567), isitsc's 1SCF
    test (isitsc.F90:34-44: ovmax below 5 selcon and |dE| below selcon on
    two consecutive iterations; ovmax is diagg1's tiny, diagg1.F90:648), and
    the shift control (:615-628).  selcon = scfcrt (scfcri's default 1e-2).
    tidy's compression step (atoms with negligible coefficients dropped)
    runs at the top of every iteration (:221, :326); not restated: tidy's
    repacking of the storage (the LMOs carry their own spare slots),
    PLS_faulty's restart, COSMO.  occ and vir are updated in place.
    Returns a dict: escf, ee, niter, converged, history."""
    iorbs = (s.nlast - s.nfirst + 1).astype(np.int32)
    mpack, nijbo = layout(iorbs, s.coord, cutof1, cutof2)
    idg = idiag(iorbs, nijbo)
    h = dense_to_blocks(so.unpack(s.h, s.norbs), iorbs, nijbo, mpack)
    selcon = scfcrt
    thresh = 1.0e-13
    const = 1.0                          # DAMP for main-group atoms (diagg2.F90:56-63)
    bigeps = 50.0 * np.sqrt(1.0e-39)
    cap = 300 * s.norbs
    st = np.array([10.0, 1.0, 0.0, 0.0])  # diagg1's fref, safety, oldlim, tiny
    nfmo = np.zeros(len(vir[0]), np.int32)
    ifmo = np.zeros(2 * cap, np.int32)
    fmo = np.zeros(cap)
    nrejct = np.zeros(2, np.int32)
    eigs = np.zeros(len(occ[0]))
    eigv = np.zeros(len(vir[0]))
    p = density(iorbs, nijbo, occ, 0, mpack)
    f = fock(s.nat, s.coord, iorbs, nijbo, s.w, p, h)
    ee = helecz(iorbs, nijbo, p, h, f)
    escf = (ee + s.enuclr) * so.FPC9 + s.atheat
    pold = np.zeros(mpack)
    p1, p2, p3 = np.zeros(s.norbs), np.zeros(s.norbs), np.zeros(s.norbs)
    eold, niter, idiagg, shift, lstart, nhb = 0.0, 0, 0, 0.0, 0, 0
    use3, scf1, converged = True, False, False
    history = []
    while True:
        tidy(occ, iorbs, thresh)                      # iter_for_MOZYME.F90:221, :326
        tidy(vir, iorbs, thresh)
        if check_lmos(occ, iorbs) > 0.1 or check_lmos(vir, iorbs) > 0.1:
            raise RuntimeError("ERROR DETECTED IN SUBROUTINE CHECK")
        eimp(iorbs, nijbo, p, f)
        nij, eigv, eg, _ = diagg1(iorbs, nijbo, f, p, occ, vir, idiagg, st, nfmo, ifmo, fmo, cap)
        if eg is not None:
            eigs = eg
        ovmax = float(st[3])
        diagg2(iorbs, occ, vir, ifmo, fmo, nij, eigs, eigv, idiagg, [const, shift, thresh, st[3], bigeps], nrejct)
        p = density(iorbs, nijbo, occ, 0, mpack)
        idiagg += 1
        niter += 1
        nhb_ij = 0
        if niter % 3 == 0 and nhb < 4:
            nhb += 1
            nhb_ij, hif, hfm = hbonds(iorbs, nijbo, f, p, occ, vir, HB_LIMITS[nhb - 1], cap)
            if nhb_ij:
                diagg2(iorbs, occ, vir, hif, hfm, nhb_ij, eigs, eigv, idiagg,
                       [const, shift, thresh, st[3], bigeps], nrejct)
                if idiagg % 2 == 1:
                    idiagg += 1
        if use3:
            cnvgz(p, pold, p1, p2, p3, niter, idg)
        f = fock(s.nat, s.coord, iorbs, nijbo, s.w, p, h)
        ee = helecz(iorbs, nijbo, p, h, f)
        escf = (ee + s.enuclr) * so.FPC9 + s.atheat
        de = escf - eold
        eold = escf
        if abs(de) > 9999.0:
            de = 0.0
        if trace:
            history.append(dict(niter=niter, escf=escf, de=de, ovmax=ovmax, nij=nij, hb=nhb_ij, shift=shift))
        ok = ovmax < 5.0 * selcon and abs(de) < selcon
        if (ok and scf1) or niter > itrmax:
            if niter > 3:
                converged = niter <= itrmax
                break
        scf1 = ok
        if use3:
            if niter % 3 == 2 and abs(de) < 0.1:
                use3, lstart, shift = False, niter, 0.0
        elif de > 0.0 and shift < 11.0 and niter > lstart + 2:
            shift += 2.0
            lstart = niter
    return dict(escf=escf, ee=ee, niter=niter, converged=converged, history=history)


def hcore(nat, coord, iorbs, nijbo, mpack: int, nw_max: int):
    """hcore_for_MOZYME (MOZYME/hcore_for_MOZYME.F90, molecular, mode 0): H on
    the pair blocks, W of the stored pairs (dense W order, far pairs left
    out), enuclr.  Stored pairs get the full integrals (h1elec, rotate);
    pairs between cutof2 and cutof1 outer2's monopole + dipole terms, pairs
    beyond cutof1 outer1's feathered point charge."""
    L = _lib()
    if not hasattr(L, "_mz_hcore_bound"):
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
        i64p = np.ctypeslib.ndpointer(np.int64, flags="C")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
        L.orc_mz_hcore.argtypes = [ctypes.c_int, i32p, f64p, i64p, f64p, f64p, ctypes.POINTER(ctypes.c_double)]
        L.orc_mz_hcore.restype = ctypes.c_longlong
        L._mz_hcore_bound = True
    h = np.zeros(mpack)
    w = np.zeros(nw_max)
    en = ctypes.c_double()
    nw = L.orc_mz_hcore(len(nat), np.ascontiguousarray(nat, np.int32), np.ascontiguousarray(coord, np.float64).ravel(),
                        np.ascontiguousarray(nijbo.ravel()), h, w, ctypes.byref(en))
    return h, w[:nw], en.value
