"""Per-step device entry points on torch CUDA tensors (float64, contiguous).

Thin wrappers over the mb_*_dev symbols; torch only provides the device
memory and the current stream.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import MbAtomsDev, check, lib


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: torch.Tensor):
    assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()
    return ctypes.c_void_p(t.data_ptr())


class Atoms:
    """Device atom layout from 1-based nfirst/nlast."""

    def __init__(self, nfirst, nlast):
        nf = np.ascontiguousarray(nfirst, dtype=np.int32)
        nl = np.ascontiguousarray(nlast, dtype=np.int32)
        self.s = MbAtomsDev()
        check(lib().mb_atoms_create(int(nf.size), nf.ctypes.data, nl.ctypes.data, ctypes.byref(self.s)))

    def __del__(self):
        try:
            lib().mb_atoms_destroy(ctypes.byref(self.s))
        except Exception:
            pass


def fock2(atoms: Atoms, f, h, ptot, pa, w, shift: float = 0.0, use_shift: bool = False) -> None:
    check(lib().mb_fock2_dev(ctypes.byref(atoms.s), _ptr(f), _ptr(h), _ptr(ptot), _ptr(pa), _ptr(w),
                             float(shift), int(use_shift), _stream()))


def helect(n: int, p, h, f) -> float:
    out = torch.zeros(1, dtype=torch.float64, device=p.device)
    check(lib().mb_helect_dev(n, _ptr(p), _ptr(h), _ptr(f), _ptr(out), _stream()))
    return float(out.item())


def cnvg(norbs: int, pnew, p, p1, niter: int) -> float:
    pl = torch.zeros(1, dtype=torch.float64, device=p.device)
    check(lib().mb_cnvg_dev(norbs, _ptr(pnew), _ptr(p), _ptr(p1), niter, _ptr(pl), _stream()))
    return float(pl.item())


class Pulay:
    """Device histories and host state of Pulay's converger for one density
    (the fppf, fock, emat, lfock, nfock, start arguments of
    pulay(f, p, n, fppf, fock, emat, lfock, nfock, msize, start, pl),
    SCF/pulay.F90:16).  ``step(f, p)`` extrapolates f in place and returns pl."""

    def __init__(self, n: int, npulay: int = 10, device="cuda"):
        self.n = n
        self.linear = n * (n + 1) // 2
        self.mfock = npulay
        self.fppf = torch.zeros(npulay * self.linear, dtype=torch.float64, device=device)
        self.fock = torch.zeros(npulay * self.linear, dtype=torch.float64, device=device)
        self.emat = np.zeros((npulay + 1) * (npulay + 1))   # column-major, ld npulay + 1
        nb = int(lib().mb_pulay_ws_bytes(n))
        self.ws = torch.empty(nb // 8 + 32, dtype=torch.float64, device=device)
        self.lfock = ctypes.c_int(0)
        self.nfock = ctypes.c_int(0)
        self.start = ctypes.c_int(1)

    def step(self, f, p) -> float:
        pl = ctypes.c_double(0.0)
        base = self.ws.data_ptr()
        ws = ctypes.c_void_p((base + 255) & ~255)
        check(lib().mb_pulay_ws(self.n, _ptr(f), _ptr(p), _ptr(self.fppf), _ptr(self.fock), self.mfock,
                                self.emat.ctypes.data, self.mfock + 1, ctypes.byref(self.lfock),
                                ctypes.byref(self.nfock), ctypes.byref(self.start), ctypes.byref(pl), ws,
                                _stream()))
        return pl.value


def density(c, nocc: int, occ: float = 2.0):
    """c: (n, n) column-major, i.e. a torch tensor whose .T is contiguous."""
    n = c.shape[0]
    ct = c.t().contiguous() if not c.t().is_contiguous() else c.t()
    p = torch.empty(n * (n + 1) // 2, dtype=torch.float64, device=c.device)
    check(lib().mb_density_dev(n, nocc, float(occ), ctypes.c_void_p(ct.data_ptr()), n, _ptr(p), _stream()))
    return p


def eigh_packed(fpacked):
    """Full eigensolve; adds i*1e-10 to the packed diagonal in place like the
    reference.  Returns (C column-major as a (n, n) tensor C[i, k], eigs)."""
    mp = fpacked.numel()
    n = int((np.sqrt(8 * mp + 1) - 1) / 2)
    cT = torch.empty((n, n), dtype=torch.float64, device=fpacked.device)  # cT[k, i] = C[i, k]
    e = torch.empty(n, dtype=torch.float64, device=fpacked.device)
    check(lib().mb_eigh_packed_dev(n, _ptr(fpacked), _ptr(cT), _ptr(e), _stream()))
    return cT.t(), e


def pseudo_diag(fpacked, cT, eigs, nocc: int) -> int:
    """cT[k, i] = C[i, k] (column-major C as a row-major tensor); rotated in place."""
    n = cT.shape[0]
    nrot = ctypes.c_longlong(0)
    check(lib().mb_pseudo_diag_dev(n, nocc, _ptr(fpacked), _ptr(cT), _ptr(eigs), ctypes.byref(nrot), _stream()))
    return nrot.value


def dgemm(transa: str, transb: str, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc) -> None:
    check(lib().mb_dgemm_dev(transa.encode(), transb.encode(), m, n, k, alpha, _ptr(a), lda, _ptr(b), ldb, beta,
                             _ptr(c), ldc, _stream()))


def _aligned_ws(nbytes: int, device, align: int = 1024):
    buf = torch.empty(nbytes + align, dtype=torch.uint8, device=device)
    return buf, ctypes.c_void_p((buf.data_ptr() + align - 1) & ~(align - 1))


def matmul_split(a, b, alpha: float = 1.0):
    """alpha * a @ b for row-major float64 CUDA tensors through the
    split-precision tensor-core GEMM (mb_gemm_split_ws)."""
    m, k = a.shape
    k2, n = b.shape
    assert k == k2
    a = a.contiguous()
    b = b.contiguous()
    c = torch.empty((m, n), dtype=torch.float64, device=a.device)
    nb = int(lib().mb_gemm_split_ws_bytes(n, m, k))
    buf, ws = _aligned_ws(nb, a.device)
    err = torch.zeros(1, dtype=torch.int32, device=a.device)
    # row-major C = A B is column-major C^T = B^T A^T
    check(lib().mb_gemm_split_ws(b"N", b"N", n, m, k, float(alpha), _ptr(b), n, _ptr(a), k, 0.0, _ptr(c), n, ws,
                                 nb, ctypes.c_void_p(err.data_ptr()), _stream()))
    if int(err.item()) != 0:
        raise RuntimeError("tensor-core GEMM pipeline wait expired")
    del buf
    return c


def density_split(c, nocc: int, occ: float = 2.0):
    """density() with the split-precision tensor-core product."""
    n = c.shape[0]
    ct = c.t().contiguous() if not c.t().is_contiguous() else c.t()
    p = torch.empty(n * (n + 1) // 2, dtype=torch.float64, device=c.device)
    nb = int(lib().mb_density_split_ws_bytes(n, nocc))
    buf, ws = _aligned_ws(nb, c.device)
    err = torch.zeros(1, dtype=torch.int32, device=c.device)
    check(lib().mb_density_split_ws(n, nocc, float(occ), ctypes.c_void_p(ct.data_ptr()), n, _ptr(p), ws, nb,
                                    ctypes.c_void_p(err.data_ptr()), _stream()))
    if int(err.item()) != 0:
        raise RuntimeError("tensor-core GEMM pipeline wait expired")
    del buf
    return p
