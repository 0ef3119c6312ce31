"""Failure detection without a GPU fault: the tcgen05 GEMM's bounded
mbarrier wait (the primitive every wait of that kernel goes through) is made
to run out on a barrier nothing arrives at; it must give up after its limit,
report it, and leave the context usable."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mopac_gpu_b200 import build
    build.build()


@pytest.mark.parametrize("limit_ms", [1, 20])
def test_bounded_wait_gives_up_and_reports(limit_ms):
    from mopac_gpu_b200._lib import check, lib
    out = torch.zeros(2, dtype=torch.int64, device="cuda")
    check(lib().mb_selftest_bounded_wait(limit_ms * 1000000, ctypes.c_void_p(out.data_ptr()), None))
    gave_up, waited_ns = out.cpu().tolist()
    assert gave_up == 1
    assert limit_ms * 1e6 <= waited_ns < limit_ms * 1e6 + 50e6
    # the context still works: a density build right after
    n, k = 64, 20
    c = torch.as_tensor(np.linalg.qr(np.random.default_rng(0).normal(size=(n, n)))[0].ravel(order="F"),
                        device="cuda")
    p = torch.empty(n * (n + 1) // 2, dtype=torch.float64, device="cuda")
    check(lib().mb_density_dev(n, k, 2.0, ctypes.c_void_p(c.data_ptr()), n, ctypes.c_void_p(p.data_ptr()), None))
    torch.cuda.synchronize()
    assert np.isfinite(p.cpu().numpy()).all()
