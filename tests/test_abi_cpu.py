"""CPU checks of the C ABI: the library builds for sm_100a, loads, and exports
every function include/mopac_b200.h declares.  No compute is called."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    txt = open(os.path.join(ROOT, "include", "mopac_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?(?:void|int|double|size_t|long long|char\s*\*|const char\s*\*)\s*\**\s*(\w+)\s*\(",
                       txt, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def libpath():
    from mopac_gpu_b200 import build
    return build.build()


def test_header_declares_reference_symbols():
    names = _declared_functions()
    for ref in ["call_gemm_cublas", "call_syrk_cublas", "call_gemm_cublas_2gpu", "call_syrk_cublas_2gpu",
                "mopac_cuda_dsyevd", "call_rot_cuda_gpu", "call_rot_cuda_2gpu_gpu", "getGPUInfo", "setDevice",
                "set_mozyme_gpu_pair", "create_handle", "destroy_handle", "mopac_cuda_destroy_resources",
                "fock2_", "helect_", "cnvg_", "density_for_gpu_", "eigenvectors_lapack_", "diag_for_gpu_",
                "mb_scf_run", "mb_ctx_create", "mb_fock2_dev", "mb_eigh_packed_dev"]:
        assert ref in names, ref


def test_library_exports_every_declared_symbol(libpath):
    names = _declared_functions()
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if l.strip()}
    missing = [n for n in names if n not in exported]
    assert not missing, missing


def test_library_loads_and_reports_version(libpath):
    L = ctypes.CDLL(libpath)
    L.mb_version.restype = ctypes.c_int
    assert L.mb_version() >= 100


def test_python_loader_binds_all_signatures(libpath):
    from mopac_gpu_b200 import _lib
    L = _lib.lib()
    for name in _lib.SIGNATURES:
        assert getattr(L, name) is not None


def test_bad_arguments_fail_loudly_without_gpu_work(libpath):
    from mopac_gpu_b200 import _lib
    L = _lib.lib()
    h = ctypes.c_void_p()
    import numpy as np
    nat = np.array([9], np.int32)  # fluorine: outside this build
    rc = L.mb_ctx_create(1, nat.ctypes.data, None, ctypes.byref(h))
    assert rc == 5
    assert b"element" in L.mb_last_error()


def test_plain_c_client_links_and_runs(libpath, tmp_path):
    """tests/c_abi_client.c, built with gcc against include/mopac_b200.h and
    the in-tree library alone, runs its host-only checks."""
    exe = tmp_path / "c_abi_client"
    libdir = os.path.dirname(libpath)
    r = subprocess.run(["gcc", "-std=c11", "-O1", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "c_abi_client.c"), "-L", libdir, "-lmopac_b200",
                        f"-Wl,-rpath,{libdir}", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe), str(tmp_path / "x.den")], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, (run.returncode, run.stderr)
    assert "c_abi_client ok" in run.stdout


def test_mozyme_fock_without_elements_refuses_cutoffs_below_the_feathering_distance(libpath):
    """A 6 A cutoff puts far pairs inside PM7's point-charge feathering, whose
    terms need the elements: mb_mz_fock_dev (no atomic numbers) refuses it
    before it touches the device (the pointers below are never
    dereferenced); mb_mz_fock_nat_dev takes it."""
    from mopac_gpu_b200._lib import MbMzLayout
    L = ctypes.CDLL(libpath)
    L.mb_mz_fock_dev.restype = ctypes.c_int
    L.mb_last_error.restype = ctypes.c_char_p
    lay = MbMzLayout()
    lay.numat = 3
    lay.cutof1, lay.cutof2 = 6.0, 5.9 ** 2
    fake = ctypes.c_void_p(256)
    rc = L.mb_mz_fock_dev(ctypes.byref(lay), fake, fake, fake, fake, fake, fake, None)
    assert rc == 5  # MB_ERR_UNSUPPORTED
    assert b"cutof2" in L.mb_last_error()


def test_fock2_workspace_is_checked_before_any_gpu_work(libpath):
    """mb_fock2_ws refuses a missing, short or misaligned workspace with
    MB_ERR_ARG before it touches the device; the size is 10 numat^2 doubles
    of staging plus the two atom lists and a 256-byte header."""
    from mopac_gpu_b200._lib import MbAtomsDev
    L = ctypes.CDLL(libpath)
    L.mb_fock2_ws_bytes.restype = ctypes.c_size_t
    L.mb_fock2_ws_bytes.argtypes = [ctypes.c_int]
    L.mb_last_error.restype = ctypes.c_char_p
    numat = 5
    need = L.mb_fock2_ws_bytes(numat)
    assert need == 256 + 2 * 256 + 8 * 10 * numat * numat
    assert L.mb_fock2_ws_bytes(0) == 0
    at = MbAtomsDev()
    at.numat = numat
    fake = ctypes.c_void_p(4096)
    args = [ctypes.byref(at), fake, fake, fake, fake, fake, ctypes.c_double(0.0), ctypes.c_int(0)]
    L.mb_fock2_ws.restype = ctypes.c_int
    assert L.mb_fock2_ws(*args, None, ctypes.c_size_t(need), None) == 1
    assert L.mb_fock2_ws(*args, fake, ctypes.c_size_t(need - 8), None) == 1
    assert b"mb_fock2_ws_bytes" in L.mb_last_error()
    assert L.mb_fock2_ws(*args, ctypes.c_void_p(4096 + 8), ctypes.c_size_t(need), None) == 1
    assert b"aligned" in L.mb_last_error()


def test_bounded_wait_selftest_checks_its_limit_before_any_gpu_work(libpath):
    L = ctypes.CDLL(libpath)
    L.mb_selftest_bounded_wait.restype = ctypes.c_int
    L.mb_selftest_bounded_wait.argtypes = [ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_void_p]
    fake = ctypes.c_void_p(4096)
    assert L.mb_selftest_bounded_wait(0, fake, None) == 1
    assert L.mb_selftest_bounded_wait(200000000, fake, None) == 1
    assert L.mb_selftest_bounded_wait(1000, None, None) == 1


def test_mozyme_layout_refuses_non_finite_coordinates_before_any_gpu_work(libpath):
    """A NaN or infinite coordinate is refused before the pair search (the
    cell grid needs finite extents) and before any device allocation."""
    import numpy as np
    from mopac_gpu_b200._lib import MbMzLayout
    L = ctypes.CDLL(libpath)
    L.mb_mz_layout_create.restype = ctypes.c_int
    L.mb_last_error.restype = ctypes.c_char_p
    iorbs = np.array([4, 1, 1], np.int32)
    for bad in (np.nan, np.inf):
        xyz = np.array([0.0, 0.0, 0.0, 0.96, 0.0, 0.0, bad, 0.9, 0.0])
        lay = MbMzLayout()
        rc = L.mb_mz_layout_create(3, iorbs.ctypes.data, xyz.ctypes.data, ctypes.c_double(100.0),
                                   ctypes.c_double(98.0), ctypes.byref(lay), None)
        assert rc == 1  # MB_ERR_ARG
        assert b"non-finite" in L.mb_last_error()
