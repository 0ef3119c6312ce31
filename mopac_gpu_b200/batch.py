"""Batched SCF over many small molecules (one persistent launch).

``Batch(molecules)`` takes a list of (atomic numbers, coordinates) pairs,
computes every molecule's integrals on the GPU, and ``run()`` performs every
molecule's SCF (iter, SCF/iter.F90, full diagonalisation each iteration) in
one launch, replayed from a CUDA graph; it returns the heats of formation as
iter computes them.  ``autotune()`` picks the launch configuration
(back-transformation block size, CTAs per SM) by timing them on the batch.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import ScfOpts, check, lib


class Batch:
    def __init__(self, molecules):
        nats = [np.asarray(m[0], np.int32) for m in molecules]
        xyzs = [np.asarray(m[1], np.float64).reshape(-1, 3) for m in molecules]
        self.nmol = len(nats)
        self.numat = np.array([len(n) for n in nats], np.int32)
        nat = np.ascontiguousarray(np.concatenate(nats), np.int32)
        xyz = np.ascontiguousarray(np.concatenate(xyzs), np.float64)
        self._h = ctypes.c_void_p()
        check(lib().mb_batch_create(self.nmol, self.numat.ctypes.data, nat.ctypes.data, xyz.ctypes.data,
                                    ctypes.byref(self._h)))
        self.norbs = [int(np.where(n == 1, 1, 4).sum()) for n in nats]
        self._nats = nats

    def run(self, scfcrt: float = 1.0e-4, itrmax: int = 2000):
        o = ScfOpts()
        lib().mb_scf_opts_default(ctypes.byref(o))
        o.scfcrt = scfcrt
        o.itrmax = itrmax
        escf = np.zeros(self.nmol)
        niter = np.zeros(self.nmol, np.int32)
        conv = np.zeros(self.nmol, np.int32)
        t = ctypes.c_double()
        check(lib().mb_batch_run(self._h, ctypes.byref(o), escf.ctypes.data, niter.ctypes.data, conv.ctypes.data,
                                 ctypes.byref(t)))
        return escf, niter, conv.astype(bool), t.value

    def set_config(self, nb: int = 8, per_sm: int = 0):
        check(lib().mb_batch_set_config(self._h, int(nb), int(per_sm)))

    def config(self):
        nb, grid = ctypes.c_int(), ctypes.c_int()
        check(lib().mb_batch_get_config(self._h, ctypes.byref(nb), ctypes.byref(grid)))
        return nb.value, grid.value

    def autotune(self, scfcrt: float = 1.0e-4, itrmax: int = 2000):
        """Returns (block size, CTAs per SM (0 = all that fit), best ms)."""
        o = ScfOpts()
        lib().mb_scf_opts_default(ctypes.byref(o))
        o.scfcrt = scfcrt
        o.itrmax = itrmax
        nb, per, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        check(lib().mb_batch_autotune(self._h, ctypes.byref(o), ctypes.byref(nb), ctypes.byref(per),
                                      ctypes.byref(ms)))
        return nb.value, per.value, ms.value

    PHASES = ("fock", "energy", "householder", "bisection", "inverse_iteration", "back_transform", "density",
              "cnvg")

    def set_phase_timing(self, on: bool = True):
        check(lib().mb_batch_set_phase_timing(self._h, int(on)))

    def phase_cycles(self) -> dict:
        """SM cycles per phase summed over all CTAs of the last run."""
        out = np.zeros(len(self.PHASES), np.uint64)
        check(lib().mb_batch_phase_cycles(self._h, out.ctypes.data))
        return dict(zip(self.PHASES, out.tolist()))

    def density(self, m: int) -> np.ndarray:
        n = self.norbs[m]
        p = np.empty(n * (n + 1) // 2)
        check(lib().mb_batch_get_density(self._h, int(m), p.ctypes.data))
        return p

    def hw(self, m: int):
        """(H packed, W, enuclr) of molecule m as the batch computed them."""
        lim = np.where(self._nats[m] == 1, 1, 10)
        cum = np.concatenate([[0], np.cumsum(lim)[:-1]])
        n2 = int((lim * (cum + lim)).sum())
        n = self.norbs[m]
        h = np.empty(n * (n + 1) // 2)
        w = np.empty(n2)
        en = ctypes.c_double()
        check(lib().mb_batch_get_hw(self._h, int(m), h.ctypes.data, w.ctypes.data, ctypes.byref(en)))
        return h, w, en.value

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().mb_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
