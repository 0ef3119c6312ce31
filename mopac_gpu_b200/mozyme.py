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

from ._lib import MbMzLayout, MbMzLmos, check, lib


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


def fock(layout: Layout, coord, w, ptot, h, out=None):
    """buildf(f, partf, 0): F = H + G(P) over the pair-block storage.  coord
    (numat x 3, Angstrom), w (the stored pairs' integrals, layout.nw), ptot
    and h: CUDA float64 tensors."""
    f = out if out is not None else torch.empty(layout.mpack, dtype=torch.float64, device="cuda")
    ws = torch.empty(int(lib().mb_mz_fock_ws_bytes(ctypes.byref(layout.s))) // 8 + 1, dtype=torch.float64,
                     device="cuda")
    c = coord.contiguous()
    check(lib().mb_mz_fock_dev(ctypes.byref(layout.s), _ptr(c), _ptr(w), _ptr(ptot), _ptr(h), _ptr(f), _ptr(ws),
                               _stream()))
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
