"""Host-side mirror of the reference's SCF entry point.

``ScfContext`` owns a device-resident SCF context (H, W, F, P, C and the
eigenvalues stay in HBM).  ``run`` is the counterpart of ``iter``
(SCF/iter.F90) for closed-shell PM7: it returns the heat of formation
``escf`` as iter computes it (kcal/mol, without the post-SCF geometry
terms), the electronic energy, and the iteration count; errors surface as
``LibraryError`` (MB_ERR_NOCONV is the reference's "UNABLE TO ACHIEVE
SELF-CONSISTENCE").
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from ._lib import ScfOpts, ScfRes, check, lib


@dataclass
class ScfResult:
    escf: float
    ee: float
    niter: int
    converged: bool
    n_full_diag: int
    n_pseudo_diag: int
    pl: float
    t_fock_ms: float
    t_diag_ms: float
    t_density_ms: float
    t_other_ms: float
    t_total_ms: float
    n_pulay: int = 0
    n_split: int = 0
    n_finish: int = 0
    dp: float = -1.0
    n_interp: int = 0        # Camp-King interpolated passes
    forced_on: bool = False  # iter forced all convergers on (niter > itrmax - 10)
    exit_split: bool = False  # exit diagonalisation solved as the occupied and virtual blocks
    exit_coupling: float = -1.0  # ||C_v^T F C_o||_F at the exit when the split was tried (eV)


class ScfContext:
    def __init__(self, nat, coord):
        self.nat = np.ascontiguousarray(nat, dtype=np.int32)
        self.coord = np.ascontiguousarray(coord, dtype=np.float64).reshape(-1, 3)
        L = lib()
        h = ctypes.c_void_p()
        check(L.mb_ctx_create(int(self.nat.shape[0]), self.nat.ctypes.data, self.coord.ctypes.data,
                              ctypes.byref(h)))
        self._h = h
        self.norbs = L.mb_ctx_norbs(h)
        self.nclose = L.mb_ctx_nclose(h)
        self.n2elec = L.mb_ctx_n2elec(h)
        self.mpack = self.norbs * (self.norbs + 1) // 2

    # -- integrals
    def hcore(self) -> None:
        check(lib().mb_ctx_hcore(self._h))

    def set_hw(self, h: np.ndarray, w: np.ndarray, enuclr: float) -> None:
        h = np.ascontiguousarray(h, dtype=np.float64)
        w = np.ascontiguousarray(w, dtype=np.float64)
        assert h.size == self.mpack and w.size == self.n2elec
        check(lib().mb_ctx_set_hw(self._h, h.ctypes.data, w.ctypes.data, float(enuclr)))

    def get_hw(self):
        h = np.empty(self.mpack)
        w = np.empty(self.n2elec)
        e = ctypes.c_double()
        check(lib().mb_ctx_get_hw(self._h, h.ctypes.data, w.ctypes.data, ctypes.byref(e)))
        return h, w, e.value

    # -- SCF
    def set_guess(self, p: np.ndarray) -> None:
        """Starting density for ``run(guess=True)`` (packed, host), entered like
        a density read with OLDENS (SCF/iter.F90:151-158)."""
        p = np.ascontiguousarray(p, dtype=np.float64)
        assert p.size == self.mpack
        check(lib().mb_ctx_set_guess(self._h, p.ctypes.data))

    def learned_guess(self, model, purify: int = 1) -> None:
        """Starting density predicted on the device by the atom-pair network
        (``guess.GuessModel``), then ``purify`` McWeeny steps; use with
        ``run(guess=True)``."""
        check(lib().mb_ctx_guess(self._h, model.handle, int(purify)))

    def run(self, pseudo: bool = False, scfcrt: float = 1.0e-4, itrmax: int = 2000, precision: int = 0,
            switch_pl: float = 1.0e-4, verbose: bool = False, pulay: bool = False,
            guess: bool = False, finish_dp: float = -1.0, finish_max: int = 40,
            shift: float | None = None, camp: bool = False) -> ScfResult:
        """finish_dp: the FP64 finish (mb_scf_opts.finish_dp): < 0 automatic
        (1e-7 with precision=1, off with precision=0), 0 off, > 0 the bound on
        the last density update max|P_k - P_(k-1)| before convergence is
        accepted.  shift: the SHIFT=n keyword (None: the default level shift;
        0: no level shift, SCF/iter.F90:131-136).  camp: the CAMP keyword
        (Camp-King's interp, mb_scf_opts.camp)."""
        o = ScfOpts()
        lib().mb_scf_opts_default(ctypes.byref(o))
        o.pseudo = int(pseudo)
        o.scfcrt = scfcrt
        o.itrmax = itrmax
        o.precision = precision
        o.switch_pl = switch_pl
        o.verbose = int(verbose)
        o.pulay = int(pulay)
        o.guess = int(guess)
        o.finish_dp = float(finish_dp)
        o.finish_max = int(finish_max)
        if shift is not None:
            o.bshift = -float(shift)
        o.camp = int(camp)
        r = ScfRes()
        check(lib().mb_scf_run(self._h, ctypes.byref(o), ctypes.byref(r)))
        return ScfResult(r.escf, r.ee, r.niter, bool(r.converged), r.n_full_diag, r.n_pseudo_diag, r.pl,
                         r.t_fock_ms, r.t_diag_ms, r.t_density_ms, r.t_other_ms, r.t_total_ms, r.n_pulay, r.n_split,
                         r.n_finish, r.dp, r.n_interp, bool(r.forced_on), bool(r.exit_split), r.exit_coupling)

    def density(self) -> np.ndarray:
        p = np.empty(self.mpack)
        check(lib().mb_ctx_get_density(self._h, p.ctypes.data))
        return p

    def gradient(self) -> np.ndarray:
        """Cartesian gradient of the SCF energy at the current density,
        (numat, 3) kcal/mol/A (dcart, forces/dcart.F90, for a molecule)."""
        g = np.empty((len(self.nat), 3))
        check(lib().mb_ctx_gradient(self._h, g.ctypes.data))
        return g

    def vectors(self):
        c = np.empty((self.norbs, self.norbs), order="F")
        e = np.empty(self.norbs)
        check(lib().mb_ctx_get_vectors(self._h, c.ctypes.data, e.ctypes.data))
        return c, e

    def fock(self) -> np.ndarray:
        f = np.empty(self.mpack)
        check(lib().mb_ctx_get_fock(self._h, f.ctypes.data))
        return f

    def device_ptrs(self):
        ps = [ctypes.c_void_p() for _ in range(6)]
        check(lib().mb_ctx_device_ptrs(self._h, *[ctypes.byref(p) for p in ps]))
        return dict(zip(["h", "w", "f", "p", "c", "eigs"], [p.value for p in ps]))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().mb_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def run_scf(nat, coord, pseudo: bool = False, **kw):
    """Integrals on the GPU, then the SCF; returns (ScfResult, context)."""
    ctx = ScfContext(nat, coord)
    ctx.hcore()
    return ctx.run(pseudo=pseudo, **kw), ctx
