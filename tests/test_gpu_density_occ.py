"""density_for_GPU with every occupation it takes (matrix/density_for_GPU.F90:
16-130, densit.F90) on the GPU against the oracle: closed shell, fractional
occupancy in the electron and the positron equivalent, one UHF spin, every
iopc form, through mb_density_occ_dev and the density_for_gpu_ shim.  The
reference's products are BLAS calls with no fixed summation order, so the
bar is 1e-12 of max|P|."""
import ctypes

import numpy as np
import pytest

from oracle import scf_oracle as so

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CASES = [
    # n, ndubl, nsingl, occ, fract, mode, iopc
    (60, 20, 20, 2.0, 0.0, 1, 4),      # closed shell, small-n kernel
    (300, 120, 120, 2.0, 0.0, 1, 5),   # closed shell, DMMA kernel
    (300, 100, 104, 2.0, 1.0, 1, 3),   # open shells, DGEMM form
    (300, 100, 104, 2.0, 1.0, 1, 6),   # the same, densit's explicit sums
    (300, 100, 180, 2.0, 0.5, 1, 3),   # positron equivalent (nsingl > n/2)
    (300, 100, 180, 2.0, 0.5, 1, 5),
    (300, 100, 180, 2.0, 0.5, 2, 3),   # mode 2: electron equivalent kept
    (301, 90, 95, 1.0, 0.5, 1, 2),     # one UHF spin, DGEMM form
    (301, 90, 90, 1.0, 0.0, 1, 5),     # one UHF spin, closed
    (200, 0, 30, 2.0, 0.7, 1, 3),      # nothing doubly occupied
]


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mopac_gpu_b200 import build
    build.build()


def _mos(n, seed):
    return np.linalg.qr(np.random.default_rng(seed).normal(size=(n, n)))[0]


@pytest.mark.parametrize("case", CASES, ids=[f"n{c[0]}_d{c[1]}_s{c[2]}_o{c[3]}_f{c[4]}_m{c[5]}_i{c[6]}" for c in CASES])
def test_density_occ_matches_the_oracle(case):
    from mopac_gpu_b200._lib import check, lib
    n, nd, ns, occ, fract, mode, iopc = case
    c = _mos(n, n + nd)
    ref = so.density_for_gpu(c, fract, nd, ns, occ, mode, iopc)
    dc = torch.as_tensor(np.asfortranarray(c).ravel(order="F"), device="cuda")
    dp = torch.full((n * (n + 1) // 2,), float("nan"), dtype=torch.float64, device="cuda")
    check(lib().mb_density_occ_dev(n, nd, ns, occ, fract, mode, iopc, ctypes.c_void_p(dc.data_ptr()), n,
                                   ctypes.c_void_p(dp.data_ptr()), None))
    got = dp.cpu().numpy()
    assert np.all(np.isfinite(got))
    np.testing.assert_allclose(got, ref, atol=1e-12 * max(1.0, np.abs(ref).max()))


def test_density_shim_takes_fractional_occupancy():
    """density_for_gpu_ (gfortran mangling, host arrays) with open shells and
    the positron equivalent, iopc 3 as iter uses it for half-electron runs."""
    from mopac_gpu_b200._lib import lib
    L = lib()
    n, nd, ns, occ, fract = 120, 40, 70, 2.0, 1.0
    c = np.asfortranarray(_mos(n, 9))
    pp = np.zeros(n * (n + 1) // 2)
    i, d = ctypes.c_int, ctypes.c_double
    ref = so.density_for_gpu(c, fract, nd, ns, occ, 1, 3)
    L.density_for_gpu_(c.ctypes.data_as(ctypes.c_void_p), ctypes.byref(d(fract)), ctypes.byref(i(nd)),
                       ctypes.byref(i(ns)), ctypes.byref(d(occ)), ctypes.byref(i(pp.size)), ctypes.byref(i(n)),
                       ctypes.byref(i(1)), pp.ctypes.data_as(ctypes.c_void_p), ctypes.byref(i(3)))
    np.testing.assert_allclose(pp, ref, atol=1e-12 * np.abs(ref).max())
