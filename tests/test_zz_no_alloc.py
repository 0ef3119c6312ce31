"""The allocation-free energy entry point against the allocating one.

mb_helect_noalloc is for callers that cannot allocate device memory where
they need the energy (a host arena owning all device memory, stream capture,
latency-bound loops).  Its scratch is a fixed array inside the library, so it
is checked here through the C ABI against mb_helect_dev on the same inputs,
twice in a row (the second call reuses the array the first one left behind).
This file is collected last so a failure here comes after every other test.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _packed_inputs(n, seed):
    rng = np.random.default_rng(seed)
    mp = n * (n + 1) // 2
    p = rng.uniform(-0.5, 1.0, mp)
    h = rng.normal(scale=10.0, size=mp)
    f = rng.normal(scale=10.0, size=mp)
    return [torch.as_tensor(x, device="cuda") for x in (p, h, f)]


@pytest.mark.parametrize("n,seed", [(96, 1), (3072, 2), (16384, 3)])
def test_noalloc_matches_allocating_helect_twice(n, seed):
    from mopac_gpu_b200._lib import lib
    L = lib()
    p, h, f = _packed_inputs(n, seed)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    out_ref = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert L.mb_helect_dev(n, p.data_ptr(), h.data_ptr(), f.data_ptr(), out_ref.data_ptr(), stream) == 0
    for _ in range(2):
        out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        rc = L.mb_helect_noalloc(n, p.data_ptr(), h.data_ptr(), f.data_ptr(), out.data_ptr(), stream)
        assert rc == 0, L.mb_last_error()
        torch.cuda.synchronize()
        ref = float(out_ref.item())
        assert abs(float(out.item()) - ref) <= 1e-12 * max(1.0, abs(ref))


def test_noalloc_rejects_oversize_without_touching_memory():
    from mopac_gpu_b200._lib import lib
    L = lib()
    rc = L.mb_helect_noalloc(16385, None, None, None, None, None)
    assert rc == 1
    assert b"16384" in L.mb_last_error()
