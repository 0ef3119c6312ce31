"""dfock2 on the device (mb_dfock2_dev and the reference-name shim dfock2_)
against the oracle's restatement of forces/dfock2.F90: bit for bit, for
every atom of molecules with heavy and light atoms."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import dfock_oracle as dfo

pytestmark = pytest.mark.gpu

CASES = {
    "water_pair": [8, 1, 1, 8, 1, 1],
    "propane": [6, 6, 6] + [1] * 8,
    "h3": [1, 1, 1],
    "co2_like": [8, 6, 8],
}


def _layout(nat):
    first, last, o = [], [], 1
    for z in nat:
        k = 1 if z == 1 else 4
        first.append(o)
        last.append(o + k - 1)
        o += k
    return first, last, o - 1


def _inputs(nat, seed):
    rng = np.random.default_rng(seed)
    first, last, n = _layout(nat)
    mp = n * (n + 1) // 2
    return first, last, n, rng.normal(size=mp), rng.normal(size=mp), rng.normal(size=mp), rng


@pytest.mark.parametrize("name", list(CASES))
def test_dfock2_device_is_bit_identical(name):
    from mopac_gpu_b200._lib import lib
    nat = CASES[name]
    first, last, n, f0, ptot, p, rng = _inputs(nat, 11)
    fi = (ctypes.c_int * len(nat))(*first)
    la = (ctypes.c_int * len(nat))(*last)
    for nati in range(1, len(nat) + 1):
        nw = int(lib().mb_dfock2_w_len(len(nat), fi, la, nati))
        _, nw_o = dfo.partner_sizes(first, last, nati)
        assert nw == nw_o
        w = rng.normal(size=nw)
        fo = f0.copy()
        dfo.dfock2(fo, ptot, p, w, first, last, nati)
        fd = torch.tensor(f0, dtype=torch.float64, device="cuda")
        td = [torch.tensor(x, dtype=torch.float64, device="cuda") for x in (ptot, p, w)]
        assert lib().mb_dfock2_dev(len(nat), fi, la, nati, fd.data_ptr(), td[0].data_ptr(), td[1].data_ptr(),
                                   td[2].data_ptr(), torch.cuda.current_stream().cuda_stream) == 0
        torch.cuda.synchronize()
        assert np.array_equal(fd.cpu().numpy(), fo), (name, nati)


def test_dfock2_shim_on_host_buffers():
    from mopac_gpu_b200._lib import lib
    nat = CASES["propane"]
    first, last, n, f0, ptot, p, rng = _inputs(nat, 12)
    fi = (ctypes.c_int * len(nat))(*first)
    la = (ctypes.c_int * len(nat))(*last)
    na = ctypes.c_int(len(nat))
    for nati in (1, 5):
        _, nw = dfo.partner_sizes(first, last, nati)
        w = rng.normal(size=nw)
        fo = f0.copy()
        dfo.dfock2(fo, ptot, p, w, first, last, nati)
        fh = f0.copy()
        ni = ctypes.c_int(nati)
        lib().dfock2_(fh.ctypes.data, ptot.ctypes.data, p.ctypes.data, w.ctypes.data, ctypes.byref(na), fi, la,
                      ctypes.byref(ni))
        assert np.array_equal(fh, fo)
