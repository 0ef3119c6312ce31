"""Electronic-state exchange with stock MOPAC.

``write_density_file`` / ``read_density_file``: the DENOUT / OLDENS restart
file of den_in_out (SCF/iter.F90:1133-1227) -- one record ``norbs, numat,
pa`` with pa the packed alpha density (P/2 for a closed shell), gfortran's
unformatted layout or list-directed text (DENOUTF).  ``save_state`` /
``load_state``: the C API's ``struct mopac_state`` (include/mopac.h:123-132)
as mopac_save / mopac_load fill and read it
(interface/mopac_api_saveload.F90:26-78).  A loaded state or density file
becomes the starting density of the next ``ScfContext.run(guess=True)``.
All of it runs in libmopac_b200.so (csrc/state_io.cu).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from ._lib import check, lib


def write_density_file(path: str, pa: np.ndarray, norbs: int, numat: int, formatted: bool = False) -> None:
    pa = np.ascontiguousarray(pa, dtype=np.float64)
    assert pa.size == norbs * (norbs + 1) // 2
    check(lib().mb_den_write(str(path).encode(), int(norbs), int(numat), pa.ctypes.data, int(formatted)))


def read_density_file(path: str, norbs: int, numat: int, formatted: bool = False):
    """Returns (pa, formatted_read)."""
    pa = np.empty(norbs * (norbs + 1) // 2)
    fmt = ctypes.c_int(int(formatted))
    check(lib().mb_den_read(str(path).encode(), int(norbs), int(numat), pa.ctypes.data, ctypes.byref(fmt)))
    return pa, bool(fmt.value)


@dataclass
class MopacState:
    """struct mopac_state: mpack (0: no state), uhf, pa, pb."""
    mpack: int = 0
    uhf: int = 0
    pa: np.ndarray | None = None
    pb: np.ndarray | None = None


def save_state(ctx) -> MopacState:
    mp, uhf = ctypes.c_int(), ctypes.c_int()
    check(lib().mb_ctx_save_state(ctx._h, ctypes.byref(mp), ctypes.byref(uhf), None))
    pa = np.empty(mp.value)
    check(lib().mb_ctx_save_state(ctx._h, ctypes.byref(mp), ctypes.byref(uhf), pa.ctypes.data))
    return MopacState(mp.value, uhf.value, pa, None)


def load_state(ctx, state: MopacState) -> None:
    pa = None if state.pa is None else np.ascontiguousarray(state.pa, np.float64)
    pb = None if state.pb is None else np.ascontiguousarray(state.pb, np.float64)
    check(lib().mb_ctx_load_state(ctx._h, int(state.mpack), int(state.uhf),
                                  None if pa is None else pa.ctypes.data, None if pb is None else pb.ctypes.data))


def denout(ctx, path: str, formatted: bool = False) -> None:
    """DENOUT: the context's current density to a restart file."""
    st = save_state(ctx)
    write_density_file(path, st.pa, ctx.norbs, len(ctx.nat), formatted)


def oldens(ctx, path: str) -> bool:
    """OLDENS: a restart file becomes the starting density (run(guess=True)).
    Returns whether the file was the formatted kind."""
    pa, fmt = read_density_file(path, ctx.norbs, len(ctx.nat))
    load_state(ctx, MopacState(pa.size, 0, pa, None))
    return fmt
