"""MOZYME sparse pair-block kernels on torch CUDA tensors.

Mirrors the reference's MOZYME routines that the SCF loop (iter_for_MOZYME,
MOZYME/iter_for_MOZYME.F90) calls on the block-sparse P, H and F:
``density`` = density_for_MOZYME, ``helecz`` = helecz, ``cnvgz`` = cnvgz.
``Layout`` is fillij's storage, ``Lmos`` the occupied LMOs of MOZYME_C.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import MbMzLayout, MbMzLmos, MzScfOpts, MzScfRes, check, lib


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: torch.Tensor):
    assert t.is_cuda and t.is_contiguous()
    return ctypes.c_void_p(t.data_ptr())


def _device_view(addr: int, count: int, typestr: str) -> torch.Tensor:
    """A torch view of library-owned device memory (no copy)."""
    class _A:
        __cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (addr, False), "version": 3,
                                    "strides": None}
    return torch.as_tensor(_A(), device="cuda")


class Layout:
    """Pair-block storage for atoms with iorbs orbitals at coord (Angstrom);
    cutof1, cutof2 squared as in fillij."""

    def __init__(self, iorbs, coord, cutof1: float, cutof2: float, want_nijbo: bool = False):
        self.iorbs = np.ascontiguousarray(iorbs, np.int32)
        c = np.ascontiguousarray(coord, np.float64).reshape(-1)
        n = self.iorbs.size
        self.nijbo = np.zeros(n * n, np.int64) if want_nijbo else None
        self.s = MbMzLayout()
        check(lib().mb_mz_layout_create(n, self.iorbs.ctypes.data, c.ctypes.data, float(cutof1), float(cutof2),
                                        ctypes.byref(self.s),
                                        self.nijbo.ctypes.data if want_nijbo else None))
        if want_nijbo:
            self.nijbo = self.nijbo.reshape(n, n)
        self.mpack = int(self.s.mpack)
        self.norbs = int(self.iorbs.sum())
        idg = np.zeros(self.norbs, np.int64)
        check(lib().mb_mz_idiag(ctypes.byref(self.s), idg.ctypes.data))
        self.idiag_host = idg
        self.idiag = torch.from_numpy(idg).cuda()

    def close(self):
        if self.s is not None:
            lib().mb_mz_layout_destroy(ctypes.byref(self.s))
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Lmos:
    """Occupied LMOs given as the reference's (ncf, nncf, icocc, ncocc, cocc)."""

    def __init__(self, layout: Layout, lmos):
        ncf, nncf, icocc, ncocc, cocc = (np.ascontiguousarray(x) for x in lmos)
        self._keep = (ncf.astype(np.int32), nncf.astype(np.int32), icocc.astype(np.int32),
                      ncocc.astype(np.int32), cocc.astype(np.float64))
        ncf, nncf, icocc, ncocc, cocc = self._keep
        self.s = MbMzLmos()
        self.numat = int(layout.iorbs.size)
        self._iorbs = layout.iorbs
        check(lib().mb_mz_lmos_create(layout.iorbs.size, layout.iorbs.ctypes.data, int(ncf.size), ncf.ctypes.data,
                                      nncf.ctypes.data, icocc.ctypes.data, ncocc.ctypes.data, cocc.ctypes.data,
                                      int(icocc.size), int(cocc.size), ctypes.byref(self.s)))

    def refresh(self):
        """Rebuild the per-atom index after diagg2 grew LMOs."""
        check(lib().mb_mz_lmos_refresh(self.numat, self._iorbs.ctypes.data, ctypes.byref(self.s)))

    def to_host(self):
        """(ncf, icocc, cocc) as they are on the device now."""
        n = int(self.s.nlmo)
        return (_device_view(self.s.ncf, n, "<i4").cpu().numpy(),
                _device_view(self.s.icocc, int(self.s.nentries), "<i4").cpu().numpy(),
                _device_view(self.s.cocc, int(self.s.ncoeff), "<f8").cpu().numpy())

    def close(self):
        if self.s is not None:
            lib().mb_mz_lmos_destroy(ctypes.byref(self.s))
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def density(layout: Layout, lmos: Lmos, mode: int = 0, partp=None, out=None):
    p = out if out is not None else torch.empty(layout.mpack, dtype=torch.float64, device="cuda")
    check(lib().mb_mz_density_dev(ctypes.byref(layout.s), ctypes.byref(lmos.s), int(mode),
                                  _ptr(partp) if partp is not None else None, _ptr(p), _stream()))
    return p


def helecz(layout: Layout, p, h, f) -> float:
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    ws = torch.empty(int(lib().mb_mz_helecz_ws_bytes()) // 8 + 1, dtype=torch.float64, device="cuda")
    check(lib().mb_mz_helecz_ws(layout.mpack, layout.norbs, _ptr(layout.idiag), _ptr(p), _ptr(h), _ptr(f),
                                _ptr(out), _ptr(ws), _stream()))
    return float(out.item())


def cnvgz(layout: Layout, pnew, p, p1, p2, p3, niter: int, use3: bool = True) -> float:
    pm = torch.zeros(1, dtype=torch.float64, device="cuda")
    ws = torch.empty(int(lib().mb_mz_cnvgz_ws_bytes()) // 8, dtype=torch.float64, device="cuda")
    check(lib().mb_mz_cnvgz_ws(layout.norbs, layout.mpack, _ptr(pnew), _ptr(p), _ptr(p1), _ptr(p2), _ptr(p3),
                               int(niter), _ptr(layout.idiag), int(use3), _ptr(pm), _ptr(ws), _stream()))
    return float(pm.item())


def hcore(layout: Layout, nat, coord):
    """hcore_for_MOZYME on the device: (h pair blocks, w stored-pair integrals,
    enuclr).  nat (int32) and coord (numat x 3, float64): CUDA tensors."""
    h = torch.empty(layout.mpack, dtype=torch.float64, device="cuda")
    w = torch.empty(int(layout.s.nw), dtype=torch.float64, device="cuda")
    en = torch.zeros(1, dtype=torch.float64, device="cuda")
    ws = torch.empty(int(lib().mb_mz_hcore_ws_bytes(ctypes.byref(layout.s))) // 8 + 1, dtype=torch.float64,
                     device="cuda")
    check(lib().mb_mz_hcore_dev(ctypes.byref(layout.s), _ptr(nat.contiguous()), _ptr(coord.contiguous()), _ptr(h),
                                _ptr(w), _ptr(en), _ptr(ws), _stream()))
    return h, w, float(en.item())


def fock(layout: Layout, coord, w, ptot, h, out=None, nat=None):
    """buildf(f, partf, 0): F = H + G(P) over the pair-block storage.  coord
    (numat x 3, Angstrom), w (the stored pairs' integrals, layout.nw), ptot
    and h: CUDA float64 tensors; nat (CUDA int32 atomic numbers) is needed
    for a cutoff below 7 A."""
    f = out if out is not None else torch.empty(layout.mpack, dtype=torch.float64, device="cuda")
    ws = torch.empty(int(lib().mb_mz_fock_ws_bytes(ctypes.byref(layout.s))) // 8 + 1, dtype=torch.float64,
                     device="cuda")
    c = coord.contiguous()
    if nat is None:
        check(lib().mb_mz_fock_dev(ctypes.byref(layout.s), _ptr(c), _ptr(w), _ptr(ptot), _ptr(h), _ptr(f),
                                   _ptr(ws), _stream()))
    else:
        check(lib().mb_mz_fock_nat_dev(ctypes.byref(layout.s), _ptr(nat.contiguous()), _ptr(c), _ptr(w), _ptr(ptot),
                                       _ptr(h), _ptr(f), _ptr(ws), _stream()))
    return f


class Diagg1:
    """diagg1's saved state (MOZYME/diagg1.F90: fref, safety, oldlim, tiny
    and the interaction list) for one SCF, on the device."""

    def __init__(self, layout: Layout, occ: Lmos, vir: Lmos, cap: int):
        self.layout, self.occ, self.vir, self.cap = layout, occ, vir, int(cap)
        self.state = np.array([10.0, 1.0, 0.0, 0.0])
        nv = int(vir.s.nlmo)
        self.nfmo = torch.zeros(nv, dtype=torch.int32, device="cuda")
        self.ifmo = torch.zeros(2 * self.cap, dtype=torch.int32, device="cuda")
        self.fmo = torch.zeros(self.cap, dtype=torch.float64, device="cuda")
        self.eigv = torch.zeros(nv, dtype=torch.float64, device="cuda")
        self.eigs = torch.zeros(int(occ.s.nlmo), dtype=torch.float64, device="cuda")
        nb = int(lib().mb_mz_diagg1_ws_bytes(ctypes.byref(layout.s), ctypes.byref(occ.s), ctypes.byref(vir.s)))
        self.ws = torch.empty(nb // 8 + 64, dtype=torch.float64, device="cuda")
        self.nij = 0

    def __call__(self, fao, p, idiagg: int):
        nij = ctypes.c_longlong(self.cap)
        done = ctypes.c_int(0)
        sumt = ctypes.c_double(0.0)
        base = (self.ws.data_ptr() + 255) & ~255
        check(lib().mb_mz_diagg1_dev(ctypes.byref(self.layout.s), ctypes.byref(self.occ.s), ctypes.byref(self.vir.s),
                                     _ptr(fao), _ptr(p), int(idiagg), self.state.ctypes.data, _ptr(self.nfmo),
                                     _ptr(self.ifmo), _ptr(self.fmo), ctypes.byref(nij), _ptr(self.eigv),
                                     _ptr(self.eigs), ctypes.byref(done), ctypes.byref(sumt), ctypes.c_void_p(base),
                                     _stream()))
        self.nij = nij.value
        return nij.value, bool(done.value), sumt.value


def diagg2(layout: Layout, occ: Lmos, vir: Lmos, d1: "Diagg1", idiagg: int, ctl, nrejct):
    """diagg2 on diagg1's list: rotates occ and vir in place.  ctl = (damping
    constant, shift, thresh, diagg1's tiny, bigeps); nrejct (int32[2]) is
    updated.  Returns (sumb, nrej)."""
    c = np.ascontiguousarray(ctl, np.float64)
    sumb = ctypes.c_double(0.0)
    nrej = ctypes.c_longlong(0)
    check(lib().mb_mz_diagg2_dev(ctypes.byref(layout.s), ctypes.byref(occ.s), ctypes.byref(vir.s), _ptr(d1.ifmo),
                                 _ptr(d1.fmo), int(d1.nij), _ptr(d1.eigs), _ptr(d1.eigv), int(idiagg),
                                 c.ctypes.data, nrejct.ctypes.data, ctypes.byref(sumb), ctypes.byref(nrej),
                                 _stream()))
    return sumb.value, nrej.value


HB_LIMITS = (1.0, 0.1, 0.01, 0.001)   # addhb's cutoffs on its first four calls


class _HbList:
    """hbonds' list in the shape diagg2 takes from Diagg1."""

    def __init__(self, ifmo, fmo, nij, eigs, eigv):
        self.ifmo, self.fmo, self.nij, self.eigs, self.eigv = ifmo, fmo, nij, eigs, eigv


def iter_for_mozyme(layout: Layout, occ: Lmos, vir: Lmos, coord, w, h, enuclr: float, atheat: float,
                    scfcrt: float = 1.0e-2, itrmax: int = 2000, cap: int | None = None, trace: bool = False,
                    nat=None):
    """The MOZYME SCF loop (MOZYME/iter_for_MOZYME.F90:218-630) for a whole
    closed-shell system on the device: density, Fock and energy of the
    starting LMOs, then per iteration tidy's compression, check, eimp, diagg
    (diagg1 + diagg2 +
    density), addhb every third iteration while fewer than four were made,
    cnvgz while the three-point extrapolation is on, buildf, helecz, isitsc's
    1SCF test and the shift control.  coord (numat x 3), w (the stored pairs'
    integrals) and h (pair blocks) are CUDA float64 tensors; occ and vir are
    updated in place.  The host sees scalars each iteration (energy, diagg1's
    tiny) and, four times per SCF, hbonds' atom-pair flags.  nat (CUDA
    int32 atomic numbers) is needed for a cutoff below 7 A.  Returns a dict:
    escf, ee, niter, converged, history, p, f."""
    fpc9 = 23.060547830619029
    n = layout.norbs
    cap = cap or 300 * n
    selcon = scfcrt
    const, thresh, bigeps = 1.0, 1.0e-13, 50.0 * np.sqrt(1.0e-39)
    D = Diagg1(layout, occ, vir, cap)
    hb_ifmo = torch.zeros(2 * cap, dtype=torch.int32, device="cuda")
    hb_fmo = torch.zeros(cap, dtype=torch.float64, device="cuda")
    norm_o = torch.empty(max(1, int(occ.s.nlmo)), dtype=torch.float64, device="cuda")
    norm_v = torch.empty(max(1, int(vir.s.nlmo)), dtype=torch.float64, device="cuda")
    nrejct = np.zeros(2, np.int32)
    L = lib()
    p = density(layout, occ, 0)
    f = fock(layout, coord, w, p, h, nat=nat)
    ee = helecz(layout, p, h, f)
    escf = (ee + enuclr) * fpc9 + atheat
    pold = torch.zeros(layout.mpack, dtype=torch.float64, device="cuda")
    p1, p2, p3 = (torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(3))
    eold, niter, idiagg, shift, lstart, nhb = 0.0, 0, 0, 0.0, 0, 0
    use3, scf1, converged = True, False, False
    history = []
    while True:
        # tidy's compression step (iter_for_MOZYME.F90:221, :326)
        check(L.mb_mz_tidy_dev(ctypes.byref(occ.s), layout.s.iorbs, thresh, _stream()))
        check(L.mb_mz_tidy_dev(ctypes.byref(vir.s), layout.s.iorbs, thresh, _stream()))
        occ.refresh()
        vir.refresh()
        eo, ev = ctypes.c_double(), ctypes.c_double()
        check(L.mb_mz_check_dev(ctypes.byref(occ.s), layout.s.iorbs, _ptr(norm_o), ctypes.byref(eo), _stream()))
        check(L.mb_mz_check_dev(ctypes.byref(vir.s), layout.s.iorbs, _ptr(norm_v), ctypes.byref(ev), _stream()))
        if eo.value > 0.1 or ev.value > 0.1:
            raise RuntimeError("ERROR DETECTED IN SUBROUTINE CHECK")
        check(L.mb_mz_eimp_dev(ctypes.byref(layout.s), _ptr(p), _ptr(f), _stream()))
        nij, _, _ = D(f, p, idiagg)
        ovmax = float(D.state[3])
        diagg2(layout, occ, vir, D, idiagg, [const, shift, thresh, D.state[3], bigeps], nrejct)
        occ.refresh()
        vir.refresh()
        p = density(layout, occ, 0)
        idiagg += 1
        niter += 1
        nhb_ij = 0
        if niter % 3 == 0 and nhb < 4:
            nhb += 1
            nn = ctypes.c_longlong(0)
            check(L.mb_mz_hbonds_dev(ctypes.byref(layout.s), ctypes.byref(occ.s), ctypes.byref(vir.s), _ptr(f),
                                     _ptr(p), HB_LIMITS[nhb - 1], cap, _ptr(hb_ifmo), _ptr(hb_fmo),
                                     ctypes.byref(nn), _stream()))
            nhb_ij = nn.value
            if nhb_ij:
                diagg2(layout, occ, vir, _HbList(hb_ifmo, hb_fmo, nhb_ij, D.eigs, D.eigv), idiagg,
                       [const, shift, thresh, D.state[3], bigeps], nrejct)
                occ.refresh()
                vir.refresh()
                if idiagg % 2 == 1:
                    idiagg += 1
        if use3:
            cnvgz(layout, p, pold, p1, p2, p3, niter, True)
        f = fock(layout, coord, w, p, h, nat=nat)
        ee = helecz(layout, p, h, f)
        escf = (ee + enuclr) * fpc9 + atheat
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
    return dict(escf=escf, ee=ee, niter=niter, converged=converged, history=history, p=p, f=f)


def scf_run(layout: Layout, occ: Lmos, vir: Lmos, coord, w, h, enuclr: float, atheat: float,
            scfcrt: float = 1.0e-2, itrmax: int = 2000, cap: int | None = None, verbose: bool = False,
            nat=None):
    """The MOZYME SCF behind its C entry (mb_mz_scf_run): the loop of
    ``iter_for_mozyme`` run by the library.  Returns a dict: escf, ee, niter,
    converged, t_total_ms, nrejected, p, f."""
    o = MzScfOpts()
    lib().mb_mz_scf_opts_default(ctypes.byref(o))
    o.scfcrt = float(scfcrt)
    o.itrmax = int(itrmax)
    o.cap = int(cap or 0)
    o.verbose = int(verbose)
    nat_d = None if nat is None else nat.contiguous()
    o.nat = None if nat_d is None else nat_d.data_ptr()
    p = torch.empty(layout.mpack, dtype=torch.float64, device="cuda")
    f = torch.empty(layout.mpack, dtype=torch.float64, device="cuda")
    r = MzScfRes()
    check(lib().mb_mz_scf_run(ctypes.byref(layout.s), layout.iorbs.ctypes.data, ctypes.byref(occ.s),
                              ctypes.byref(vir.s), _ptr(coord.contiguous()), _ptr(w), _ptr(h), float(enuclr),
                              float(atheat), ctypes.byref(o), _ptr(p), _ptr(f), ctypes.byref(r), _stream()))
    return dict(escf=r.escf, ee=r.ee, niter=r.niter, converged=bool(r.converged), t_total_ms=r.t_total_ms,
                nrejected=r.nrejected, p=p, f=f)


# ------------------------------------------------------------ starting LMOs
def _pipek_mezey(C: np.ndarray, atom_of: np.ndarray, natoms: int, sweeps: int = 200) -> np.ndarray:
    """Pipek-Mezey localisation of the columns of C (orthonormal NDDO AO
    basis): 2x2 Jacobi rotations that maximise the sum over orbitals and
    atoms of the squared atomic populations."""
    C = C.copy()
    n = C.shape[1]
    masks = [atom_of == a for a in range(natoms)]
    for _ in range(sweeps):
        largest = 0.0
        for i in range(n):
            for j in range(i + 1, n):
                A = B = 0.0
                for m in masks:
                    pii, pjj, pij = float(C[m, i] @ C[m, i]), float(C[m, j] @ C[m, j]), float(C[m, i] @ C[m, j])
                    A += pij * pij - 0.25 * (pii - pjj) ** 2
                    B += pij * (pii - pjj)
                if A * A + B * B < 1.0e-24:
                    continue
                g = 0.25 * np.arccos(-A / np.hypot(A, B)) * (1.0 if B >= 0.0 else -1.0)
                c, s = np.cos(g), np.sin(g)
                ci, cj = C[:, i].copy(), C[:, j].copy()
                C[:, i] = c * ci + s * cj
                C[:, j] = -s * ci + c * cj
                largest = max(largest, abs(g))
        if largest < 1.0e-12:
            break
    return C


def _water_frame_axes(o, h1, h2) -> np.ndarray:
    """Orthonormal axes (columns) of a water molecule: the HOH bisector, the
    H1-H2 direction, their cross product."""
    e1 = (h1 - o) + (h2 - o)
    e1 /= np.linalg.norm(e1)
    e2 = h1 - h2
    e2 -= (e2 @ e1) * e1
    e2 /= np.linalg.norm(e2)
    return np.stack([e1, e2, np.cross(e1, e2)], axis=1)


def _water_frames(o, h1, h2) -> np.ndarray:
    """_water_frame_axes for every molecule at once: (nmol, 3, 3)."""
    e1 = (h1 - o) + (h2 - o)
    e1 = e1 / np.sqrt(np.einsum("mi,mi->m", e1, e1))[:, None]
    e2 = h1 - h2
    e2 = e2 - np.einsum("mi,mi->m", e2, e1)[:, None] * e1
    e2 = e2 / np.sqrt(np.einsum("mi,mi->m", e2, e2))[:, None]
    return np.stack([e1, e2, np.cross(e1, e2)], axis=2)


def _water_lmo_arrays(C, o, h1, h2, pad_atoms: int):
    """The reference's LMO arrays (ncf, nncf, icocc, ncocc, cocc) for one
    water's localised orbitals C (6 x nl: O s, px, py, pz, H1 s, H2 s)
    carried into every molecule (O at o[m], hydrogens at h1[m], h2[m]): the s
    coefficients as they are, the p coefficients rotated from the first
    molecule's frame into each molecule's.  LMO m * nl + k lists its three
    atoms by falling weight in C[:, k], followed by pad_atoms spare slots."""
    nmol, nl = len(o), C.shape[1]
    R0 = _water_frames(o[:1], h1[:1], h2[:1])[0]
    Rm = _water_frames(o, h1, h2)                            # (nmol, 3, 3)
    q = np.einsum("ji,jk->ik", R0, C[1:4, :])                # (3, nl): frame components
    pm = np.einsum("mij,jk->mik", Rm, q)                     # (nmol, 3, nl)
    per_icocc = 3 + pad_atoms
    per_cocc = 6 + 4 * pad_atoms
    nlmo = nmol * nl
    ncf = np.full(nlmo, 3, np.int32)
    nncf = (np.arange(nlmo) * per_icocc).astype(np.int32)
    ncocc = (np.arange(nlmo) * per_cocc).astype(np.int32)
    icocc = np.zeros((nmol, nl, per_icocc), np.int32)
    cocc = np.zeros((nmol, nl, per_cocc))
    mol = np.arange(nmol)
    for k in range(nl):
        weights = np.array([np.sum(C[:4, k] ** 2), C[4, k] ** 2, C[5, k] ** 2])
        pos = 0
        for slot, a in enumerate(np.argsort(-weights, kind="stable")):
            icocc[:, k, slot] = 3 * mol + a + 1
            if a == 0:
                cocc[:, k, pos] = C[0, k]
                cocc[:, k, pos + 1:pos + 4] = pm[:, :, k]
                pos += 4
            else:
                cocc[:, k, pos] = C[3 + a, k]
                pos += 1
    return ncf, nncf, icocc.reshape(-1), ncocc, cocc.reshape(-1)


# covalent radii (A) of the bond graph that splits a system into molecules
_COVALENT = {1: 0.31, 6: 0.76, 8: 0.66}


def molecules(nat, xyz, scale: float = 1.25) -> list:
    """The molecules of a system: the connected components of its bond graph,
    atoms A and B bonded when r_AB < scale (R_A + R_B) with the covalent radii
    R of H, C and O (0.31, 0.76, 0.66 A).  Each molecule is the ascending
    array of its atoms (0-based); molecules come in order of their first
    atom."""
    nat = np.asarray(nat)
    parent = np.arange(len(nat))

    def root(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    for a, b in bonds(nat, xyz, scale):
        ra, rb = root(a), root(b)
        if ra != rb:
            parent[max(ra, rb)] = min(ra, rb)
    roots = np.array([root(a) for a in range(len(nat))])
    return [np.flatnonzero(roots == r) for r in np.unique(roots)]


def bonds(nat, xyz, scale: float = 1.25) -> np.ndarray:
    """The bond graph's edges (a, b), a < b, in ascending order: atoms closer
    than scale times the sum of their covalent radii (H 0.31, C 0.76,
    O 0.66 A)."""
    from scipy.spatial import cKDTree
    nat = np.asarray(nat)
    xyz = np.asarray(xyz, float).reshape(-1, 3)
    try:
        rad = np.array([_COVALENT[int(z)] for z in nat])
    except KeyError as e:
        raise ValueError(f"element {e} outside H, C, O") from None
    if len(nat) < 2:
        return np.zeros((0, 2), np.int64)
    pairs = cKDTree(xyz).query_pairs(r=2.0 * scale * rad.max(), output_type="ndarray")
    if len(pairs) == 0:
        return np.zeros((0, 2), np.int64)
    pairs = np.sort(pairs, axis=1)
    d = np.linalg.norm(xyz[pairs[:, 0]] - xyz[pairs[:, 1]], axis=1)
    pairs = pairs[d < scale * (rad[pairs[:, 0]] + rad[pairs[:, 1]])]
    return pairs[np.lexsort((pairs[:, 1], pairs[:, 0]))]


def _perpendicular(axis: np.ndarray) -> np.ndarray:
    """A unit vector perpendicular to the unit vector axis."""
    t = np.eye(3)[int(np.argmin(np.abs(axis)))]
    v = t - (t @ axis) * axis
    return v / np.linalg.norm(v)


def _pi_bonds(nat, nbr, valence):
    """Multiple bonds of a neutral closed-shell H, C, O Lewis structure: each
    atom's missing valence (valence - sigma bonds) is paired along its bonds,
    first where an atom has a single bonded partner with missing valence,
    then in ascending atom order.  Returns the pi bonds (a, b), a < b, a
    double bond once and a triple bond twice."""
    need = [valence[int(z)] - len(nbr[a]) for a, z in enumerate(nat)]
    if min(need, default=0) < 0:
        a = int(np.argmin(need))
        raise ValueError(f"lewis_lmos: atom {a + 1} has more bonds than its valence")
    pis = []
    while any(need):
        pick = None
        for a in range(len(nat)):
            if need[a] > 0:
                cand = [b for b in nbr[a] if need[b] > 0]
                if not cand:
                    raise ValueError(f"lewis_lmos: atom {a + 1} has no partner for a multiple bond "
                                     "(a radical or an ion)")
                if len(cand) == 1:
                    pick = (a, cand[0])
                    break
        if pick is None:
            a = next(x for x in range(len(nat)) if need[x] > 0)
            pick = (a, min(b for b in nbr[a] if need[b] > 0))
        a, b = pick
        need[a] -= 1
        need[b] -= 1
        pis.append((min(a, b), max(a, b)))
    return sorted(pis)


def lewis_lmos(nat, xyz, pad_atoms: int = 0, scale: float = 1.25):
    """Starting LMOs from the Lewis structure of a neutral closed-shell H, C, O
    system (one large molecule or many), the job makvec
    (MOZYME/makvec.F90:16-143) does, here from the bond directions rather
    than from makvec's Fock-matrix hybrids.  Bonds come from ``bonds``;
    missing valence (C 4, O 2, H 1) is paired into double and triple bonds
    (``_pi_bonds``); an atom with missing valence and no partner for it (a
    radical, an ion) raises ValueError.  Every O carries two lone pairs.

    A heavy atom's sigma hybrids point along its bonds and lone pairs: sp3
    for four of them (an O's two lone pairs complete the tetrahedron of its
    two bonds, 54.74 degrees either side of their plane, on the far side of
    their bisector), sp2 for three (a carbonyl O's lone pairs at 120 degrees
    from its bond, in the plane perpendicular to the pi orbital), sp for two;
    the remaining p orbitals carry the pi bonds, perpendicular to the sp2
    plane or to the sp axis, the same direction on both atoms of a pi bond;
    the atom's hybrids and p orbitals are orthonormalised symmetrically
    (Loewdin).  An H's hybrid is its s orbital.  A bond A-B (sigma or pi,
    A < B) gives the occupied LMO (h_A + h_B)/sqrt(2) and the virtual LMO
    (h_A - h_B)/sqrt(2) on atoms A, B; a lone pair is the occupied LMO h_A
    on its atom alone.  The LMOs are orthonormal, nclose occupied and
    norbs - nclose virtual.  They come atom by atom: the atom's sigma bonds
    to higher atoms, then its pi bonds to higher atoms, then its lone pairs.
    Returns (iorbs, occ, vir) in the reference's arrays (ncf, nncf, icocc,
    ncocc, cocc), pad_atoms spare atom slots after every LMO."""
    nat = np.asarray(nat).astype(np.int32)
    xyz = np.asarray(xyz, float).reshape(-1, 3)
    iorbs = np.where(nat == 1, 1, 4).astype(np.int32)
    edges = bonds(nat, xyz, scale)
    nbr = [[] for _ in range(len(nat))]
    for a, b in edges:
        nbr[a].append(int(b))
        nbr[b].append(int(a))
    valence = {1: 1, 6: 4, 8: 2}
    pis = _pi_bonds(nat, nbr, valence)
    if any(int(nat[a]) == 1 or int(nat[b]) == 1 for a, b in pis):
        raise ValueError("lewis_lmos: hydrogen in a multiple bond")
    npi = [0] * len(nat)
    for a, b in pis:
        npi[a] += 1
        npi[b] += 1
    unit = lambda v: v / np.linalg.norm(v)
    sdir = [[unit(xyz[b] - xyz[a]) for b in nbr[a]] for a in range(len(nat))]
    lone = [2 if z == 8 else 0 for z in nat]
    # pi directions: from the atoms whose sigma frame fixes them, then carried
    # to their partners; pdir[a] lists atom a's pi directions in use order
    pdir = [None] * len(nat)
    for a in range(len(nat)):
        ns = len(nbr[a]) + lone[a]
        if npi[a] == 0:
            continue
        if npi[a] == 1 and len(nbr[a]) >= 2:      # sp2 with two or three sigma bonds
            d = np.array(sdir[a])
            # the normal of the bonds' plane: the direction they span least
            pdir[a] = [unit(np.linalg.svd(d)[2][-1])] if len(d) > 2 else [unit(np.cross(d[0], d[1]))]
        elif npi[a] == 2 and ns == 2:               # sp: two pi orbitals around the axis
            ax = sdir[a][0]
            p1 = _perpendicular(ax)
            pdir[a] = [p1, unit(np.cross(ax, p1))]
    bond_dir = {}
    todo = list(pis)
    for _ in range(2 * len(pis) + 2):
        left = []
        for k, (a, b) in enumerate(todo):
            src = a if pdir[a] is not None else (b if pdir[b] is not None else None)
            if src is None:
                left.append((a, b))
                continue
            used = sum(1 for key in bond_dir if src in key[:2])
            d = pdir[src][min(used, len(pdir[src]) - 1)]
            other = b if src == a else a
            ax = sdir[other][nbr[other].index(src)]
            d = unit(d - (d @ ax) * ax)
            bond_dir[(a, b, len(bond_dir))] = d
            if pdir[other] is None:
                pdir[other] = [d] if npi[other] == 1 else [d, unit(np.cross(ax, d))]
        todo = left
        if not todo:
            break
    for a, b in todo:                               # neither atom fixes it: any direction off the bond
        ax = sdir[a][nbr[a].index(b)]
        d = _perpendicular(ax)
        bond_dir[(a, b, len(bond_dir))] = d
        pdir[a] = pdir[a] or [d]
        pdir[b] = pdir[b] or [d]
    half = np.arccos(-1.0 / 3.0) / 2.0
    hyb = {}   # (atom, partner) for sigma, (atom, partner, 'pi', k) for pi, (atom, -1/-2) for lone pairs
    pi_of = {}  # atom -> [(key, direction)] of its pi orbitals
    for key, d in bond_dir.items():
        a, b, k = key
        pi_of.setdefault(a, []).append(((a, b, "pi", k), d))
        pi_of.setdefault(b, []).append(((b, a, "pi", k), d))
    for a, z in enumerate(nat):
        if z == 1:
            hyb[(a, nbr[a][0])] = np.array([1.0])
            continue
        dirs = list(sdir[a])
        keys = [(a, b) for b in nbr[a]]
        ns = len(dirs) + lone[a]
        pis_a = pi_of.get(a, [])
        if lone[a]:
            if len(dirs) == 2:                      # sp3 O: lone pairs complete the tetrahedron
                bis = unit(-(dirs[0] + dirs[1]))
                nrm = unit(np.cross(dirs[0], dirs[1]))
                dirs += [np.cos(half) * bis + np.sin(half) * nrm, np.cos(half) * bis - np.sin(half) * nrm]
            elif len(dirs) == 1 and len(pis_a) == 1:  # sp2 O: lone pairs in the plane off the pi orbital
                d0, pp = dirs[0], pis_a[0][1]
                q = unit(np.cross(pp, d0))
                c120, s120 = -0.5, np.sqrt(0.75)
                dirs += [c120 * d0 + s120 * q, c120 * d0 - s120 * q]
            else:
                raise ValueError(f"lewis_lmos: oxygen {a + 1} is neither sp3 nor sp2")
            keys += [(a, -1), (a, -2)]
        if ns + len(pis_a) != 4:
            raise ValueError(f"lewis_lmos: atom {a + 1} has {ns} sigma and {len(pis_a)} pi orbitals")
        cs = np.sqrt(1.0 / ns)                      # s share of an sp^(ns-1) hybrid
        rows = [[cs, *(np.sqrt(1.0 - cs * cs) * d)] for d in dirs]
        rows += [[0.0, *d] for _, d in pis_a]
        keys += [k for k, _ in pis_a]
        v = np.array(rows)
        w, u = np.linalg.eigh(v @ v.T)
        if w.min() < 1.0e-3:
            raise ValueError(f"lewis_lmos: the orbitals of atom {a + 1} are not independent")
        h = (u @ np.diag(w ** -0.5) @ u.T) @ v
        for key, row in zip(keys, h):
            hyb[key] = row
    occ, vir = [], []
    r2 = np.sqrt(0.5)
    for a in range(len(nat)):
        pairs = [((a, b), (b, a)) for b in sorted(x for x in nbr[a] if x > a)]
        pairs += [((a, b, "pi", k), (b, a, "pi", k)) for (a2, b, k) in bond_dir if a2 == a]
        for ka, kb in pairs:
            b = ka[1]
            atoms = np.array([a, b])
            occ.append((atoms, np.concatenate([r2 * hyb[ka], r2 * hyb[kb]])))
            vir.append((atoms, np.concatenate([r2 * hyb[ka], -r2 * hyb[kb]])))
        for lp in range(lone[a]):
            occ.append((np.array([a]), hyb[(a, -1 - lp)].copy()))
    return iorbs, _pack_lmos(iorbs, occ, pad_atoms), _pack_lmos(iorbs, vir, pad_atoms)


def _kabsch(p: np.ndarray, q: np.ndarray):
    """The proper rotation R (det +1) that best maps the centred points p onto
    the centred points q (rows), and the RMS distance left."""
    u, _, vt = np.linalg.svd(p.T @ q)
    d = np.sign(np.linalg.det(vt.T @ u.T)) or 1.0
    r = vt.T @ np.diag([1.0, 1.0, d]) @ u.T
    return r, float(np.sqrt(np.mean(np.sum((p @ r.T - q) ** 2, axis=1))))


def _pack_lmos(iorbs: np.ndarray, lmos: list, pad_atoms: int):
    """The reference's LMO arrays (ncf, nncf, icocc, ncocc, cocc) for LMOs
    given as (atoms, coefficients over those atoms' orbitals in that order):
    each LMO lists its atoms by falling weight (its bond's atoms first, as
    hbonds expects), followed by pad_atoms spare atom slots."""
    nl = len(lmos)
    ncf = np.array([len(atoms) for atoms, _ in lmos], np.int32)
    ncoef = np.array([len(vec) for _, vec in lmos], np.int64)
    nncf = np.concatenate([[0], np.cumsum(ncf + pad_atoms)])[:nl].astype(np.int32)
    ncocc = np.concatenate([[0], np.cumsum(ncoef + 4 * pad_atoms)])[:nl].astype(np.int32)
    icocc = np.zeros(int(ncf.sum()) + nl * pad_atoms, np.int32)
    cocc = np.zeros(int(ncoef.sum()) + nl * 4 * pad_atoms, np.float64)
    for m, (atoms, vec) in enumerate(lmos):
        atoms = np.asarray(atoms)
        no = iorbs[atoms]
        offs = np.concatenate([[0], np.cumsum(no)])
        w = np.add.reduceat(vec * vec, offs[:-1]) if len(atoms) else np.zeros(0)
        order = np.argsort(-w, kind="stable")
        icocc[nncf[m]:nncf[m] + len(atoms)] = atoms[order] + 1
        sel = np.concatenate([np.arange(offs[k], offs[k + 1]) for k in order]) if len(atoms) else np.zeros(0, int)
        cocc[ncocc[m]:ncocc[m] + len(sel)] = vec[sel]
    return ncf, nncf, icocc, ncocc, cocc


def molecule_lmos(nat, xyz, pad_atoms: int = 0, scfcrt: float = 1.0e-8, orbitals=None, same_tol: float = 1.0e-6):
    """Starting LMOs for a system of separate H, C, O molecules (a liquid, a
    mixture, a molecular crystal): the work makvec (MOZYME/makvec.F90:16-143)
    does from a Lewis structure, done from the isolated molecules.  The
    system is split into molecules by its bond graph (``molecules``); each
    distinct molecule's SCF orbitals (this library's dense SCF on the GPU, or
    ``orbitals(nat, xyz) -> (C, nclose)`` when given) are Pipek-Mezey
    localised, occupied and virtual separately, and carried into every copy
    of that molecule: a copy has the same elements in the same order and the
    same shape up to a proper rotation (RMS <= same_tol A after the best
    rotation); its LMOs keep the s coefficients and rotate the p ones.  A
    molecule with no copy earlier in the system gets its own SCF.  LMOs come
    molecule by molecule; an LMO lists all atoms of its molecule by falling
    weight and is followed by pad_atoms spare atom slots for diagg2 to grow
    it.  Returns (iorbs, occ, vir) in the reference's arrays (ncf, nncf,
    icocc, ncocc, cocc)."""
    nat = np.asarray(nat).astype(np.int32)
    xyz = np.asarray(xyz, float).reshape(-1, 3)
    if np.any((nat != 1) & (nat != 6) & (nat != 8)):
        raise ValueError("molecule_lmos: elements outside H, C, O")
    iorbs = np.where(nat == 1, 1, 4).astype(np.int32)

    def scf_orbitals(zn, r):
        if orbitals is not None:
            return orbitals(zn, r)
        from .scf import ScfContext
        ctx = ScfContext(zn, r)
        try:
            ctx.hcore()
            ctx.run(pseudo=False, scfcrt=scfcrt, finish_dp=1.0e-10, finish_max=200)
            c, _ = ctx.vectors()
            return c, ctx.nclose
        finally:
            ctx.close()

    templates = []  # (elements, centred coordinates, localised occupied, localised virtual)
    occ, vir = [], []
    for atoms in molecules(nat, xyz):
        zn, r = nat[atoms], xyz[atoms]
        centred = r - r.mean(axis=0)
        rot = None
        for tz, tc, tocc, tvir in templates:
            if len(tz) == len(zn) and np.array_equal(tz, zn):
                R, rms = _kabsch(tc, centred)
                if rms <= same_tol:
                    rot, lo, lv = R, tocc, tvir
                    break
        if rot is None:
            c, nclose = scf_orbitals(zn, r)
            atom_of = np.repeat(np.arange(len(atoms)), iorbs[atoms])
            lo = _pipek_mezey(c[:, :nclose], atom_of, len(atoms)) if nclose > 0 else c[:, :0]
            lv = _pipek_mezey(c[:, nclose:], atom_of, len(atoms)) if nclose < c.shape[0] else c[:, :0]
            templates.append((zn.copy(), centred, lo, lv))
            rot = np.eye(3)
        # the p rows of every heavy atom rotate with the molecule
        prow = np.concatenate([[0], np.cumsum(iorbs[atoms])])[:-1][iorbs[atoms] == 4]
        for src, dst in ((lo, occ), (lv, vir)):
            v = src.copy()
            for o in prow:
                v[o + 1:o + 4, :] = rot @ src[o + 1:o + 4, :]
            for k in range(v.shape[1]):
                dst.append((atoms, v[:, k]))
    return iorbs, _pack_lmos(iorbs, occ, pad_atoms), _pack_lmos(iorbs, vir, pad_atoms)


def water_lmos(nat, xyz, pad_atoms: int = 0, scfcrt: float = 1.0e-8):
    """Starting LMOs for (H2O)_n, atoms given as O, H, H per molecule: the work
    makvec (MOZYME/makvec.F90:16-143) does from a Lewis structure, done here
    from the isolated molecule -- two O-H bonds and two lone pairs occupied,
    two O-H antibonds virtual -- as the SCF orbitals of one water (this
    library's dense SCF on the GPU), Pipek-Mezey localised, then carried into
    every molecule's orientation (s coefficients unchanged, p coefficients
    rotated with the molecule).  The molecules must share one rigid internal
    geometry (checked to 1e-8 A).  Each LMO lists its atoms by falling weight
    (its bond's atoms first, as hbonds expects) and is followed by pad_atoms
    spare atom slots for diagg2 to grow it.  Returns (iorbs, occ, vir) in the
    reference's arrays (ncf, nncf, icocc, ncocc, cocc)."""
    from .scf import ScfContext
    nat = np.asarray(nat)
    xyz = np.asarray(xyz, float).reshape(-1, 3)
    nmol = len(nat) // 3
    if len(nat) != 3 * nmol or np.any(nat[0::3] != 8) or np.any(nat[1::3] != 1) or np.any(nat[2::3] != 1):
        raise ValueError("water_lmos: atoms must come as O, H, H per molecule")
    o, h1, h2 = xyz[0::3], xyz[1::3], xyz[2::3]
    geo = np.stack([np.linalg.norm(h1 - o, axis=1), np.linalg.norm(h2 - o, axis=1),
                    np.linalg.norm(h1 - h2, axis=1)], axis=1)
    if np.abs(geo - geo[0]).max() > 1.0e-8:
        raise ValueError("water_lmos: the molecules do not share one rigid geometry")
    ctx = ScfContext(nat[:3], xyz[:3])
    ctx.hcore()
    ctx.run(pseudo=False, scfcrt=scfcrt, finish_dp=1.0e-10, finish_max=200)
    c, _ = ctx.vectors()
    ctx.close()
    atom_of = np.array([0, 0, 0, 0, 1, 2])
    loc = [_pipek_mezey(c[:, :4], atom_of, 3), _pipek_mezey(c[:, 4:6], atom_of, 3)]
    iorbs = np.where(nat == 1, 1, 4).astype(np.int32)
    out = [_water_lmo_arrays(C, o, h1, h2, pad_atoms) for C in loc]
    return iorbs, out[0], out[1]
