"""Pulay's converger (SCF/pulay.F90, matrix/osinv.F90).

CPU: the oracle's osinv against numpy and against the library's host
restatement (bit-identical: both follow the same Gauss-Jordan steps), and
the oracle's Pulay SCF against the pinned default SCF at convergence.
GPU: one step at a time against the oracle (commutator history, B matrix,
extrapolated F), the Fortran shim, and whole SCFs with pulay on.
Tolerances: history entries and F 1e-10 relative to their scale (the
commutator goes through an FP64 GEMM whose summation order differs from
BLAS), heats 1e-4 kcal/mol, density 1e-6.
"""
import ctypes

import numpy as np
import pytest

from oracle import scf_oracle as so
from tests.helpers import oracle_system, small_systems

SYSTEMS = small_systems()


def _rand_sym_packed(rng, n, scale=1.0):
    a = rng.normal(size=(n, n)) * scale
    return so.pack(0.5 * (a + a.T))


# ------------------------------------------------------------------ CPU
@pytest.mark.parametrize("n", [1, 2, 3, 6, 11])
def test_oracle_osinv_inverts(n):
    rng = np.random.default_rng(n)
    a = rng.normal(size=(n, n)) + n * np.eye(n)
    ev = list(a.T.ravel())              # column-major flat
    d = so.osinv(ev, n)
    inv = np.array(ev).reshape(n, n).T
    np.testing.assert_allclose(inv, np.linalg.inv(a), rtol=1e-12, atol=1e-12)
    det = np.linalg.det(a)
    if abs(det) < 1e9:
        assert d == pytest.approx(det, rel=1e-10)
    else:                                # the running product is clamped at 1e10
        assert d <= 1e10


def test_oracle_osinv_singular_returns_zero():
    a = np.ones((3, 3))
    ev = list(a.ravel())
    assert so.osinv(ev, 3) == 0.0


def test_oracle_osinv_bordered_b_matrix():
    # the shape pulay inverts: [[B, -1], [-1^T, 0]], B scaled so B(l,l) = 1
    rng = np.random.default_rng(7)
    v = rng.normal(size=(4, 30))
    b = v @ v.T
    b /= b[2, 2]
    e = np.zeros((5, 5))
    e[:4, :4] = b
    e[4, :4] = e[:4, 4] = -1.0
    ev = list(e.ravel())
    so.osinv(ev, 5)
    coeffs = -np.array(ev[4 * 5:4 * 5 + 4])
    assert coeffs.sum() == pytest.approx(1.0, abs=1e-12)
    np.testing.assert_allclose(np.array(ev).reshape(5, 5).T, np.linalg.inv(e), atol=1e-10)


def test_library_osinv_bit_identical_to_oracle():
    from mopac_gpu_b200._lib import lib
    L = lib()
    rng = np.random.default_rng(3)
    for n in (1, 2, 5, 11):
        a = rng.normal(size=(n, n))
        ev = list(a.T.ravel())
        d0 = so.osinv(ev, n)
        buf = np.ascontiguousarray(a.T.ravel())
        d1 = L.mb_osinv(buf.ctypes.data, n)
        assert d1 == d0
        assert np.array_equal(buf, np.array(ev))
    sing = np.ones(9)
    assert L.mb_osinv(sing.ctypes.data, 3) == 0.0


def test_oracle_commutator_is_pf_minus_fp():
    rng = np.random.default_rng(1)
    n = 7
    p, f = _rand_sym_packed(rng, n), _rand_sym_packed(rng, n)
    c = so.commutator_packed(p, f, n)
    P, F = so.unpack(p, n), so.unpack(f, n)
    m = P @ F - F @ P
    r, cc = so.tri_index(n)
    np.testing.assert_allclose(c, m[cc, r], atol=1e-13)
    assert np.all(c[so.diag_index(n)] == 0.0)


@pytest.mark.parametrize("name", ["water16", "propane"])
@pytest.mark.parametrize("pseudo", [False, True])
def test_oracle_pulay_scf_reaches_pinned_state(name, pseudo):
    nat, xyz = SYSTEMS[name]
    s = oracle_system(nat, xyz)
    ref = so.iter_scf(s)
    r = so.iter_scf(s, pseudo=pseudo, pulay_on=True)
    assert r.converged
    assert abs(r.escf - ref.escf) < 2e-4
    np.testing.assert_allclose(r.p, ref.p, atol=2e-4)


# ------------------------------------------------------------------ GPU
def _need_gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize("n", [5, 40, 97])
def test_pulay_steps_match_oracle(n):
    """Twelve steps (wrapping the 10-entry history) with converging F, P."""
    torch = _need_gpu()
    from mopac_gpu_b200.kernels import Pulay
    rng = np.random.default_rng(100 + n)
    st = so.PulayState(n)
    dev = Pulay(n)
    f0, p0 = _rand_sym_packed(rng, n), _rand_sym_packed(rng, n, 0.3)
    for it in range(12):
        damp = 0.5 ** it
        f = f0 + damp * _rand_sym_packed(rng, n, 0.1)
        p = p0 + damp * _rand_sym_packed(rng, n, 0.1)
        fo = f.copy()
        pl_o = so.pulay(st, fo, p)
        fd = torch.from_numpy(f.copy()).cuda()
        pd = torch.from_numpy(p.copy()).cuda()
        pl_d = dev.step(fd, pd)
        torch.cuda.synchronize()
        assert (dev.lfock.value, dev.nfock.value, bool(dev.start.value)) == (st.lfock, st.nfock, st.start)
        assert pl_d == pytest.approx(pl_o, rel=1e-10)
        np.testing.assert_allclose(dev.fppf.cpu().numpy(), st.fppf, atol=1e-12 * max(1.0, np.abs(st.fppf).max()))
        np.testing.assert_array_equal(dev.fock.cpu().numpy(), st.fock)
        np.testing.assert_allclose(fd.cpu().numpy(), fo, rtol=0, atol=1e-9 * np.abs(fo).max())


@pytest.mark.gpu
def test_pulay_fortran_shim_matches_oracle():
    torch = _need_gpu()
    from mopac_gpu_b200._lib import lib
    L = lib()
    n = 23
    lin = n * (n + 1) // 2
    rng = np.random.default_rng(5)
    st = so.PulayState(n)
    fppf = np.zeros(10 * lin)
    fock = np.zeros(10 * lin)
    emat = np.zeros(11 * 11)
    lfock, nfock, start = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(1)
    nn, msize = ctypes.c_int(n), ctypes.c_int(10 * lin)
    f0, p0 = _rand_sym_packed(rng, n), _rand_sym_packed(rng, n, 0.3)
    for it in range(4):
        f = f0 + 0.5 ** it * _rand_sym_packed(rng, n, 0.1)
        p = p0 + 0.5 ** it * _rand_sym_packed(rng, n, 0.1)
        fo = f.copy()
        pl_o = so.pulay(st, fo, p)
        fs = f.copy()
        pl = ctypes.c_double()
        L.pulay_(fs.ctypes.data, p.ctypes.data, ctypes.byref(nn), fppf.ctypes.data, fock.ctypes.data,
                 emat.ctypes.data, ctypes.byref(lfock), ctypes.byref(nfock), ctypes.byref(msize),
                 ctypes.byref(start), ctypes.byref(pl))
        assert (lfock.value, nfock.value) == (st.lfock, st.nfock)
        assert pl.value == pytest.approx(pl_o, rel=1e-10)
        np.testing.assert_array_equal(fock, st.fock)
        np.testing.assert_allclose(fs, fo, atol=1e-9 * np.abs(fo).max())


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["water16", "propane", "co2_1scf"])
@pytest.mark.parametrize("pseudo", [False, True])
def test_pulay_scf_matches_oracle(name, pseudo):
    _need_gpu()
    from mopac_gpu_b200 import ScfContext
    nat, xyz = SYSTEMS[name]
    s = oracle_system(nat, xyz)
    ref = so.iter_scf(s, pseudo=pseudo, pulay_on=True)
    ctx = ScfContext(nat, xyz)
    ctx.set_hw(s.h, s.w, s.enuclr)
    r = ctx.run(pseudo=pseudo, pulay=True)
    p = ctx.density()
    _, e = ctx.vectors()
    ctx.close()
    assert r.converged and ref.converged
    assert r.n_pulay > 0
    assert abs(r.niter - ref.niter) <= 2
    assert abs(r.escf - ref.escf) < 1e-4
    np.testing.assert_allclose(p, ref.p, atol=1e-6)
    np.testing.assert_allclose(e, ref.eigs, atol=1e-5)
