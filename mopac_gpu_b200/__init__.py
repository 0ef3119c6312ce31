"""mopac_gpu_b200 -- B200 (sm_100a) build of MOPAC's semiempirical SCF hot path.

The compute lives in libmopac_b200.so (hand-written CUDA behind a C ABI, see
include/mopac_b200.h; the reference-named bind(C) symbols are reached through
``lib()``).  This package is the host-side mirror of the reference's SCF
entry points:
  ``ScfContext``  iter on the device (dense PM7 closed-shell SCF);
  ``batch``       many small molecules in one persistent launch;
  ``mozyme``      MOZYME's sparse-block kernels and its SCF loop;
  ``guess``       the learned initial guess (atom-pair network, its training);
  ``state``       DENOUT/OLDENS restart files and mopac_state;
  ``kernels``     per-step entry points on device buffers;
  ``replicas``    molecule sharding over ranks for multi-GPU runs.
"""
from ._lib import lib, LibraryError, MB_OK  # noqa: F401
from .scf import ScfContext, ScfResult, run_scf  # noqa: F401
from . import workloads  # noqa: F401

__all__ = ["lib", "LibraryError", "ScfContext", "ScfResult", "run_scf", "workloads"]
