"""DENOUT / OLDENS restart files and the mopac_state record (CPU parts: the
file format through the C ABI; no GPU work).  The unformatted layout is
gfortran's sequential record, built here byte by byte with struct to pin it."""
import os
import struct

import numpy as np
import pytest

from mopac_gpu_b200 import LibraryError
from mopac_gpu_b200.state import read_density_file, write_density_file


@pytest.fixture(scope="module", autouse=True)
def _lib():
    from mopac_gpu_b200 import build
    build.build()


def _pa(norbs, seed=0):
    rng = np.random.default_rng(seed)
    return rng.normal(size=norbs * (norbs + 1) // 2) * 0.3


def test_unformatted_layout_is_gfortrans_record(tmp_path):
    norbs, numat = 6, 3
    pa = _pa(norbs)
    f = tmp_path / "x.den"
    write_density_file(f, pa, norbs, numat)
    raw = f.read_bytes()
    n = 8 + 8 * pa.size
    want = struct.pack("<iii", n, norbs, numat) + pa.astype("<f8").tobytes() + struct.pack("<i", n)
    assert raw == want
    back, fmt = read_density_file(f, norbs, numat)
    assert not fmt and np.array_equal(back, pa)


def test_formatted_round_trip_is_exact_and_detected(tmp_path):
    norbs, numat = 10, 4
    pa = _pa(norbs, 1)
    f = tmp_path / "x.den"
    write_density_file(f, pa, norbs, numat, formatted=True)
    txt = f.read_text().split()
    assert txt[0] == "10" and txt[1] == "4"
    back, fmt = read_density_file(f, norbs, numat, formatted=False)  # tries unformatted first, falls back
    assert fmt and np.array_equal(back, pa)


def test_fortran_list_directed_text_with_d_exponents_and_repeats(tmp_path):
    norbs, numat = 2, 2
    f = tmp_path / "x.den"
    f.write_text("   2   2\n 0.5D+00, 2*1.25E-01\n")
    back, fmt = read_density_file(f, norbs, numat, formatted=True)
    assert fmt and np.array_equal(back, [0.5, 0.125, 0.125])


def test_file_for_another_system_is_refused(tmp_path):
    f = tmp_path / "x.den"
    write_density_file(f, _pa(6), 6, 3)
    with pytest.raises(LibraryError, match="does not match current data set"):
        read_density_file(f, 10, 4)       # larger system: header first, like the Fortran read
    with pytest.raises(LibraryError, match="does not match current data set"):
        read_density_file(f, 4, 2)        # smaller system


def test_missing_or_corrupt_file(tmp_path):
    with pytest.raises(LibraryError, match="missing or corrupt"):
        read_density_file(tmp_path / "none.den", 6, 3)
    f = tmp_path / "bad.den"
    f.write_bytes(os.urandom(7))
    with pytest.raises(LibraryError, match="missing or corrupt"):
        read_density_file(f, 6, 3)
    g = tmp_path / "short.den"
    raw = bytearray(struct.pack("<iii", 8 + 8 * 21, 6, 3) + b"\0" * 40)
    g.write_bytes(bytes(raw))                  # truncated record
    with pytest.raises(LibraryError, match="missing or corrupt"):
        read_density_file(g, 6, 3)
