"""ctypes binding of libmopac_b200.so.

The library is built in-tree (``python -m mopac_gpu_b200.build``).  Loading
fails loudly when it is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmopac_b200.so")

MB_OK = 0
ERRORS = {1: "MB_ERR_ARG", 2: "MB_ERR_CUDA", 3: "MB_ERR_NOCONV", 4: "MB_ERR_TIMEOUT",
          5: "MB_ERR_UNSUPPORTED", 6: "MB_ERR_NUMERIC", 7: "MB_ERR_NOMEM"}


class LibraryError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class MbAtomsDev(ctypes.Structure):
    _fields_ = [("numat", ctypes.c_int), ("first", ctypes.c_void_p), ("nor", ctypes.c_void_p),
                ("lim", ctypes.c_void_p), ("wrow", ctypes.c_void_p), ("cum", ctypes.c_void_p)]


class MbMzLayout(ctypes.Structure):
    _fields_ = [("numat", ctypes.c_int), ("mpack", ctypes.c_longlong), ("npairs", ctypes.c_longlong),
                ("iorbs", ctypes.c_void_p), ("pair_ptr", ctypes.c_void_p), ("pair_i", ctypes.c_void_p),
                ("pair_j", ctypes.c_void_p), ("pair_off", ctypes.c_void_p), ("pair_woff", ctypes.c_void_p),
                ("nw", ctypes.c_longlong), ("nbr_ptr", ctypes.c_void_p), ("nbr_atom", ctypes.c_void_p),
                ("nbr_entry", ctypes.c_void_p), ("cutof1", ctypes.c_double), ("cutof2", ctypes.c_double),
                ("first", ctypes.c_void_p), ("norbs", ctypes.c_int)]


class MbMzLmos(ctypes.Structure):
    _fields_ = [("nlmo", ctypes.c_int), ("atom_ptr", ctypes.c_void_p), ("atom_lmo", ctypes.c_void_p),
                ("atom_coff", ctypes.c_void_p), ("cocc", ctypes.c_void_p), ("ncf", ctypes.c_void_p),
                ("nncf", ctypes.c_void_p), ("icocc", ctypes.c_void_p), ("ncocc", ctypes.c_void_p),
                ("nentries", ctypes.c_longlong), ("ncoeff", ctypes.c_longlong)]


class MzScfOpts(ctypes.Structure):
    _fields_ = [("scfcrt", ctypes.c_double), ("itrmax", ctypes.c_int), ("cap", ctypes.c_longlong),
                ("verbose", ctypes.c_int), ("nat", ctypes.c_void_p)]


class MzScfRes(ctypes.Structure):
    _fields_ = [("escf", ctypes.c_double), ("ee", ctypes.c_double), ("niter", ctypes.c_int),
                ("converged", ctypes.c_int), ("t_total_ms", ctypes.c_double), ("nrejected", ctypes.c_longlong)]


class ScfOpts(ctypes.Structure):
    _fields_ = [("pseudo", ctypes.c_int), ("itrmax", ctypes.c_int), ("scfcrt", ctypes.c_double),
                ("precision", ctypes.c_int), ("switch_pl", ctypes.c_double), ("verbose", ctypes.c_int),
                ("pulay", ctypes.c_int), ("guess", ctypes.c_int), ("finish_dp", ctypes.c_double),
                ("finish_max", ctypes.c_int), ("bshift", ctypes.c_double), ("camp", ctypes.c_int)]


class ScfRes(ctypes.Structure):
    _fields_ = [("escf", ctypes.c_double), ("ee", ctypes.c_double), ("niter", ctypes.c_int),
                ("converged", ctypes.c_int), ("n_full_diag", ctypes.c_int), ("n_pseudo_diag", ctypes.c_int),
                ("pl", ctypes.c_double), ("t_fock_ms", ctypes.c_double), ("t_diag_ms", ctypes.c_double),
                ("t_density_ms", ctypes.c_double), ("t_other_ms", ctypes.c_double), ("t_total_ms", ctypes.c_double),
                ("n_pulay", ctypes.c_int), ("n_split", ctypes.c_int), ("n_finish", ctypes.c_int),
                ("dp", ctypes.c_double), ("n_interp", ctypes.c_int), ("forced_on", ctypes.c_int),
                ("exit_split", ctypes.c_int), ("exit_coupling", ctypes.c_double)]


_lib = None

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_LL = ctypes.c_longlong
_C = ctypes.c_char

SIGNATURES = {
    "mb_version": ([], _I),
    "mb_launch_count": ([], _LL),
    "mb_kstats_enable": ([_I], None),
    "mb_kstats_read": ([_I, ctypes.POINTER(_LL), ctypes.POINTER(_D)], _I),
    "mb_last_error": ([], ctypes.c_char_p),
    "mb_scf_opts_default": ([ctypes.POINTER(ScfOpts)], None),
    "mb_ctx_create": ([_I, _P, _P, ctypes.POINTER(_P)], _I),
    "mb_ctx_destroy": ([_P], _I),
    "mb_ctx_norbs": ([_P], _I),
    "mb_ctx_n2elec": ([_P], _LL),
    "mb_ctx_nclose": ([_P], _I),
    "mb_ctx_hcore": ([_P], _I),
    "mb_ctx_set_hw": ([_P, _P, _P, _D], _I),
    "mb_ctx_get_hw": ([_P, _P, _P, ctypes.POINTER(_D)], _I),
    "mb_scf_run": ([_P, ctypes.POINTER(ScfOpts), ctypes.POINTER(ScfRes)], _I),
    "mb_ctx_get_density": ([_P, _P], _I),
    "mb_ctx_get_vectors": ([_P, _P, _P], _I),
    "mb_ctx_get_fock": ([_P, _P], _I),
    "mb_ctx_device_ptrs": ([_P] + [ctypes.POINTER(_P)] * 6, _I),
    "mb_ctx_atoms_dev": ([_P, ctypes.POINTER(MbAtomsDev)], _I),
    "mb_atoms_create": ([_I, _P, _P, ctypes.POINTER(MbAtomsDev)], _I),
    "mb_atoms_destroy": ([ctypes.POINTER(MbAtomsDev)], _I),
    "mb_fock2_dev": ([ctypes.POINTER(MbAtomsDev), _P, _P, _P, _P, _P, _D, _I, _P], _I),
    "mb_fock2_ws_bytes": ([_I], ctypes.c_size_t),
    "mb_fock2_ws": ([ctypes.POINTER(MbAtomsDev), _P, _P, _P, _P, _P, _D, _I, _P, ctypes.c_size_t, _P], _I),
    "mb_helect_dev": ([_I, _P, _P, _P, _P, _P], _I),
    "mb_helect_noalloc": ([_I, _P, _P, _P, _P, _P], _I),
    "mb_cnvg_dev": ([_I, _P, _P, _P, _I, _P, _P], _I),
    "mb_density_dev": ([_I, _I, _D, _P, _I, _P, _P], _I),
    "mb_density_occ_dev": ([_I, _I, _I, _D, _D, _I, _I, _P, _I, _P, _P], _I),
    "mb_selftest_bounded_wait": ([ctypes.c_ulonglong, _P, _P], _I),
    "mb_ctx_gradient": ([_P, _P], _I),
    "mb_dcart_ws_bytes": ([_I], ctypes.c_size_t),
    "mb_dcart_dev": ([_P, _P, ctypes.POINTER(MbAtomsDev), _I, _P, _P, _P, ctypes.c_size_t, _P], _I),
    "mb_pulay_ws_bytes": ([_I], ctypes.c_size_t),
    "mb_pulay_ws": ([_I, _P, _P, _P, _P, _I, _P, _I, _P, _P, _P, _P, _P, _P], _I),
    "mb_osinv": ([_P, _I], _D),
    "mb_batch_create": ([_I, _P, _P, _P, ctypes.POINTER(_P)], _I),
    "mb_batch_destroy": ([_P], _I),
    "mb_batch_nmol": ([_P], _I),
    "mb_batch_run": ([_P, ctypes.POINTER(ScfOpts), _P, _P, _P, ctypes.POINTER(_D)], _I),
    "mb_batch_get_density": ([_P, _I, _P], _I),
    "mb_batch_set_phase_timing": ([_P, _I], _I),
    "mb_batch_phase_cycles": ([_P, _P], _I),
    "mb_batch_get_hw": ([_P, _I, _P, _P, ctypes.POINTER(_D)], _I),
    "mb_batch_set_config": ([_P, _I, _I], _I),
    "mb_batch_get_config": ([_P, ctypes.POINTER(_I), ctypes.POINTER(_I)], _I),
    "mb_batch_autotune": ([_P, ctypes.POINTER(ScfOpts), ctypes.POINTER(_I), ctypes.POINTER(_I),
                           ctypes.POINTER(_D)], _I),
    "mb_mz_layout_create": ([_I, _P, _P, _D, _D, ctypes.POINTER(MbMzLayout), _P], _I),
    "mb_mz_layout_destroy": ([ctypes.POINTER(MbMzLayout)], _I),
    "mb_mz_idiag": ([ctypes.POINTER(MbMzLayout), _P], _I),
    "mb_mz_lmos_create": ([_I, _P, _I, _P, _P, _P, _P, _P, _LL, _LL, ctypes.POINTER(MbMzLmos)], _I),
    "mb_mz_lmos_refresh": ([_I, _P, ctypes.POINTER(MbMzLmos)], _I),
    "mb_mz_lmos_refresh_dev": ([_I, _P, ctypes.POINTER(MbMzLmos), _P], _I),
    "mb_mz_diagg2_dev": ([ctypes.POINTER(MbMzLayout), ctypes.POINTER(MbMzLmos), ctypes.POINTER(MbMzLmos), _P, _P,
                          _LL, _P, _P, _I, _P, _P, ctypes.POINTER(_D), ctypes.POINTER(_LL), _P], _I),
    "mb_mz_lmos_destroy": ([ctypes.POINTER(MbMzLmos)], _I),
    "mb_mz_density_dev": ([ctypes.POINTER(MbMzLayout), ctypes.POINTER(MbMzLmos), _I, _P, _P, _P], _I),
    "mb_mz_fock_ws_bytes": ([ctypes.POINTER(MbMzLayout)], ctypes.c_size_t),
    "mb_mz_diagg1_ws_bytes": ([ctypes.POINTER(MbMzLayout), ctypes.POINTER(MbMzLmos), ctypes.POINTER(MbMzLmos)],
                              ctypes.c_size_t),
    "mb_mz_diagg1_dev": ([ctypes.POINTER(MbMzLayout), ctypes.POINTER(MbMzLmos), ctypes.POINTER(MbMzLmos), _P, _P,
                          _I, _P, _P, _P, _P, ctypes.POINTER(_LL), _P, _P, ctypes.POINTER(_I),
                          ctypes.POINTER(_D), _P, _P], _I),
    "mb_mz_fock_dev": ([ctypes.POINTER(MbMzLayout), _P, _P, _P, _P, _P, _P, _P], _I),
    "mb_mz_fock_nat_dev": ([ctypes.POINTER(MbMzLayout)] + [_P] * 8, _I),
    "mb_mz_helecz_ws_bytes": ([], ctypes.c_size_t),
    "mb_mz_helecz_ws": ([_LL, _I, _P, _P, _P, _P, _P, _P, _P], _I),
    "mb_mz_cnvgz_ws_bytes": ([], ctypes.c_size_t),
    "mb_mz_cnvgz_ws": ([_I, _LL, _P, _P, _P, _P, _P, _I, _P, _I, _P, _P, _P], _I),
    "mb_mz_hcore_ws_bytes": ([ctypes.POINTER(MbMzLayout)], ctypes.c_size_t),
    "mb_mz_hcore_dev": ([ctypes.POINTER(MbMzLayout), _P, _P, _P, _P, _P, _P, _P], _I),
    "mb_mz_check_dev": ([ctypes.POINTER(MbMzLmos), _P, _P, ctypes.POINTER(_D), _P], _I),
    "mb_mz_eimp_dev": ([ctypes.POINTER(MbMzLayout), _P, _P, _P], _I),
    "mb_mz_scf_opts_default": ([ctypes.POINTER(MzScfOpts)], None),
    "mb_atheat": ([_I, _P], _D),
    "mb_mz_tidy_dev": ([ctypes.POINTER(MbMzLmos), _P, _D, _P], _I),
    "mb_mz_scf_run": ([ctypes.POINTER(MbMzLayout), _P, ctypes.POINTER(MbMzLmos), ctypes.POINTER(MbMzLmos), _P, _P,
                       _P, _D, _D, ctypes.POINTER(MzScfOpts), _P, _P, ctypes.POINTER(MzScfRes), _P], _I),
    "mb_mz_hbonds_dev": ([ctypes.POINTER(MbMzLayout), ctypes.POINTER(MbMzLmos), ctypes.POINTER(MbMzLmos), _P, _P,
                          _D, _LL, _P, _P, ctypes.POINTER(_LL), _P], _I),
    "mb_gemm_split_ws_bytes": ([_I, _I, _I], ctypes.c_size_t),
    "mb_gemm_split_ws": ([_C, _C, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I, _P, ctypes.c_size_t, _P, _P], _I),
    "mb_density_split_ws_bytes": ([_I, _I], ctypes.c_size_t),
    "mb_density_split_ws": ([_I, _I, _D, _P, _I, _P, _P, ctypes.c_size_t, _P, _P], _I),
    "mb_eigh_packed_dev": ([_I, _P, _P, _P, _P], _I),
    "mb_eigh_ws_bytes": ([_I], ctypes.c_size_t),
    "mb_eigh_ws": ([_I, _P, _I, _P, _P, _P, _P, _P], _I),
    "mb_pseudo_diag_dev": ([_I, _I, _P, _P, _P, ctypes.POINTER(_LL), _P], _I),
    "mb_dgemm_dev": ([_C, _C, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I, _P], _I),
    "call_gemm_cublas": ([_C, _C, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I], None),
    "call_syrk_cublas": ([_C, _C, _I, _I, _D, _P, _I, _D, _P, _I], None),
    "call_gemm_cublas_2gpu": ([_C, _C, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I], None),
    "call_syrk_cublas_2gpu": ([_C, _C, _I, _I, _D, _P, _I, _D, _P, _I], None),
    "mopac_cuda_dsyevd": ([_I, _P, _I, _P, _P], None),
    "call_rot_cuda_gpu": ([_P, _P, _P, _P, _P, _I, _I, _I, _D, _D], None),
    "call_rot_cuda_2gpu_gpu": ([_P, _P, _P, _P, _P, _I, _I, _I, _D, _D], None),
    "getGPUInfo": ([_P] * 9, None),
    "setDevice": ([_I, _P], None),
    "set_mozyme_gpu_pair": ([_I, _I], None),
    "create_handle": ([], None),
    "destroy_handle": ([], None),
    "mopac_cuda_destroy_resources": ([], None),
    "fock2_": ([_P] * 10, None),
    "dfock2_": ([_P] * 8, None),
    "mb_dfock2_w_len": ([_I, _P, _P, _I], ctypes.c_longlong),
    "mb_dfock2_dev": ([_I, _P, _P, _I, _P, _P, _P, _P, _P], _I),
    "helect_": ([_P] * 4, _D),
    "cnvg_": ([_P] * 5, None),
    "mb_set_norbs_": ([_P], None),
    "pulay_": ([_P] * 11, None),
    "mb_set_npulay_": ([_P], None),
    "density_for_gpu_": ([_P] * 10, None),
    "eigenvectors_lapack_": ([_P] * 4, None),
    "diag_for_gpu_": ([_P] * 6, None),
    "mb_mz_bind_system_": ([_P] * 8, _I),
    "mb_mz_bind_lmos_": ([_P] * 19, _I),
    "mb_mz_bind_controls_": ([_P, _P], _I),
    "density_for_mozyme_": ([_P] * 4, None),
    "buildf_": ([_P] * 3, None),
    "diagg_": ([_P] * 6, None),
    "mb_ctx_set_guess": ([_P, _P], _I),
    "mb_den_write": ([ctypes.c_char_p, _I, _I, _P, _I], _I),
    "mb_den_read": ([ctypes.c_char_p, _I, _I, _P, ctypes.POINTER(_I)], _I),
    "mb_ctx_save_state": ([_P, ctypes.POINTER(_I), ctypes.POINTER(_I), _P], _I),
    "mb_ctx_load_state": ([_P, _I, _I, _P, _P], _I),
    "mb_ctx_guess": ([_P, _P, _I], _I),
    "mb_guess_purify_ws_bytes": ([_I], ctypes.c_size_t),
    "mb_guess_purify_dev": ([_I, _P, _I, _P, _P], _I),
    "mb_guess_purify_split_dev": ([_I, _P, _I, _P, _P, ctypes.c_size_t, _P, _P], _I),
    "mb_guess_blob_floats": ([], ctypes.c_size_t),
    "mb_guess_model_create": ([_P, ctypes.POINTER(_P)], _I),
    "mb_guess_model_destroy": ([_P], _I),
    "mb_guess_pairs_dev": ([_I, _P, _P, _D, _P, _I, _P, _P, _P, _P, _P], _I),
    "mb_guess_features_ws_bytes": ([_I], ctypes.c_size_t),
    "mb_guess_features_dev": ([_I, _P, _P, _I, _P, _P, _P, _P, _P, _P], _I),
    "mb_guess_ws_create": ([ctypes.POINTER(_P)], _I),
    "mb_guess_ws_destroy": ([_P], _I),
    "mb_guess_predict_density_ws": ([_P, _I, _P, _P, _P, _P, _I, _P, _P, _P], _I),
    "mb_guess_normalize_dev": ([_P, _I, _I, _P, _P, _P], _I),
    "mb_guess_norm_targets_dev": ([_P, _I, _I, _P, _P, _P], _I),
    "mb_guess_forward_dev": ([_P, _I, _I, _P, _P, _P, _P], _I),
    "mb_guess_assemble_dev": ([_P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P], _I),
    "mb_guess_targets_dev": ([_I, _P, _P, _P, _P, _P, _P, _P, _P, _P], _I),
    "mb_guess_predict_density_dev": ([_P, _I, _P, _P, _P, _P, _I, _P, _P], _I),
    "mb_guess_trainer_create": ([_P, _I, ctypes.POINTER(_P)], _I),
    "mb_guess_trainer_destroy": ([_P], _I),
    "mb_guess_trainer_model": ([_P], _P),
    "mb_guess_trainer_set_norm": ([_P, _I, _P, _P, _P, _P], _I),
    "mb_guess_trainer_step": ([_P, _I, _I, _P, _P, ctypes.c_float, _I, ctypes.POINTER(_D), _P], _I),
    "mb_guess_trainer_get": ([_P, _P, _P], _I),
}


def lib():
    """Load libmopac_b200.so (built in-tree); raise if it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `python -m mopac_gpu_b200.build` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != MB_OK:
        raise LibraryError(rc, lib().mb_last_error().decode(errors="replace"))
