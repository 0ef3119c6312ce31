"""mopac_gpu_b200 -- B200 (sm_100a) build of MOPAC's semiempirical SCF hot path.

The compute lives in libmopac_b200.so (hand-written CUDA behind a C ABI, see
include/mopac_b200.h).  This package is the host-side mirror of the
reference's SCF entry points: ``ScfContext`` runs ``iter`` on the device,
``kernels`` exposes the per-step entry points on device buffers, and
``compat`` calls the reference-named bind(C) symbols with host arrays.
"""
from ._lib import lib, LibraryError, MB_OK  # noqa: F401
from .scf import ScfContext, ScfResult, run_scf  # noqa: F401
from . import workloads  # noqa: F401

__all__ = ["lib", "LibraryError", "ScfContext", "ScfResult", "run_scf", "workloads"]
