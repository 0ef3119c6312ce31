"""The drop-in boundary through the reference's own signatures.

Every symbol a Fortran build of the reference binds -- the bind(C) names of
src/gpu/cuda_wrappers.cu (call_gemm_cublas :192, call_syrk_cublas :229,
mopac_cuda_dsyevd :469, call_rot_cuda_gpu :547) and the routines iter calls
by reference (fock2, density_for_GPU, eigenvectors_LAPACK, diag_for_GPU,
helect, cnvg) -- is called here through ctypes on host buffers, exactly as
the Fortran caller would, and compared with the CPU oracle.  Bit-identical
where the product kernel follows the reference's operation order (Fock,
rotations, extrapolation), FP64 rounding tolerances for the GEMMs and the
eigensolver.
"""
import ctypes

import numpy as np
import pytest

from oracle import scf_oracle as so
from tests.helpers import mixed_density, oracle_system, small_systems

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
SYSTEMS = small_systems()


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _L():
    from mopac_gpu_b200._lib import lib
    return lib()


def _p(a):
    return a.ctypes.data


def _i(v):
    return ctypes.byref(ctypes.c_int(int(v)))


def _d(v):
    return ctypes.byref(ctypes.c_double(float(v)))


@pytest.mark.parametrize("name", ["water16", "propane", "co2_1scf"])
def test_fock2_shim_is_the_oracle_fock_build(name):
    """fock2(f, ptot, p, w, wj, wk, numat, nfirst, nlast, mode) (SCF/fock2.F90:16):
    f arrives holding H and leaves with the two-electron terms added."""
    nat, xyz = SYSTEMS[name]
    s = oracle_system(nat, xyz)
    p = mixed_density(s)
    pa = np.ascontiguousarray(p * 0.5)
    ref = s.h.copy()
    so.fock2(s, ref, p, pa)
    f = s.h.copy()
    nfirst = np.ascontiguousarray(s.nfirst, np.int32)
    nlast = np.ascontiguousarray(s.nlast, np.int32)
    _L().fock2_(_p(f), _p(p), _p(pa), _p(s.w), _p(s.w), _p(s.w), _i(s.numat), _p(nfirst), _p(nlast), _i(2))
    assert np.array_equal(f, ref)


def test_density_shim_matches_the_oracle():
    """density_for_GPU(c, fract, ndubl, nsingl, occ, mpack, norbs, mode, pp, iopc)
    (matrix/density_for_GPU.F90:16) for a closed shell: P = 2 C_occ C_occ^T."""
    rng = np.random.default_rng(4)
    n, k = 131, 77
    c = np.asfortranarray(np.linalg.qr(rng.normal(size=(n, n)))[0])
    pp = np.zeros(n * (n + 1) // 2)
    _L().density_for_gpu_(_p(c), _d(0.0), _i(k), _i(0), _d(2.0), _i(pp.size), _i(n), _i(0), _p(pp), _i(4))
    np.testing.assert_allclose(pp, so.density(c, k), atol=1e-13)


@pytest.mark.parametrize("n", [5, 96, 300])
def test_eigenvectors_lapack_shim_perturbs_xmat_like_the_reference(n):
    """eigenvectors_LAPACK(eigenvecs, xmat, eigvals, ndim) adds i*1e-10 to
    diagonal element i of xmat in place (eigenvectors_LAPACK.F90:53-55), then
    solves; the perturbed xmat must come back bit for bit."""
    rng = np.random.default_rng(n)
    a = rng.normal(size=(n, n))
    x = so.pack(a + a.T)
    ref = x.copy()
    cref, wref = so.eigenvectors_lapack(ref, n)
    vec = np.zeros((n, n), order="F")
    w = np.zeros(n)
    _L().eigenvectors_lapack_(_p(vec), _p(x), _p(w), _i(n))
    assert np.array_equal(x, ref)
    np.testing.assert_allclose(w, wref, atol=1e-10 * np.abs(wref).max())
    A = so.unpack(ref, n)
    assert np.abs(A @ vec - vec * w).max() < 1e-9 * np.abs(wref).max()
    assert np.abs(vec.T @ vec - np.eye(n)).max() < 1e-10


def test_mopac_cuda_dsyevd_overwrites_a_with_vectors():
    """mopac_cuda_dsyevd(n, A, lda, W, info) (cuda_wrappers.cu:469-505):
    'V', 'U' -- the upper triangle is read, A is overwritten by the vectors."""
    rng = np.random.default_rng(9)
    n, lda = 150, 160
    s = rng.normal(size=(n, n))
    s = s + s.T
    A = np.zeros((lda, n), order="F")
    A[:n, :] = np.triu(s)          # only the upper triangle is meaningful
    A[n:, :] = 7.0                 # rows past n must be left alone
    W = np.zeros(n)
    info = ctypes.c_int(-1)
    _L().mopac_cuda_dsyevd(n, _p(A), lda, _p(W), ctypes.byref(info))
    assert info.value == 0
    wref = np.linalg.eigvalsh(s)
    np.testing.assert_allclose(W, wref, atol=1e-10 * np.abs(wref).max())
    V = A[:n, :]
    assert np.abs(s @ V - V * W).max() < 1e-9 * np.abs(wref).max()
    assert np.all(A[n:, :] == 7.0)


@pytest.mark.parametrize("tra,trb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
def test_call_gemm_cublas_with_leading_dimensions(tra, trb):
    """call_gemm_cublas(tra, trb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)
    (cuda_wrappers.cu:192): column-major with lda/ldb/ldc larger than the rows."""
    rng = np.random.default_rng(ord(tra) * 3 + ord(trb))
    m, n, k = 70, 45, 33
    ar, ac = (k, m) if tra == "T" else (m, k)
    br, bc = (n, k) if trb == "T" else (k, n)
    A = np.asfortranarray(rng.normal(size=(ar + 3, ac)))
    B = np.asfortranarray(rng.normal(size=(br + 5, bc)))
    C = np.asfortranarray(rng.normal(size=(m + 2, n)))
    opa = A[:ar].T if tra == "T" else A[:ar]
    opb = B[:br].T if trb == "T" else B[:br]
    ref = C.copy(order="F")
    ref[:m] = 0.5 * opa @ opb - 1.5 * C[:m]
    _L().call_gemm_cublas(tra.encode(), trb.encode(), m, n, k, 0.5, _p(A), ar + 3, _p(B), br + 5, -1.5, _p(C), m + 2)
    np.testing.assert_allclose(C, ref, atol=1e-12)


@pytest.mark.parametrize("uplo,tra", [("U", "N"), ("U", "T"), ("L", "N")])
def test_call_syrk_cublas_touches_one_triangle(uplo, tra):
    """call_syrk_cublas(uplo, tra, n, k, alpha, A, lda, beta, C, ldc)
    (cuda_wrappers.cu:229): C = alpha op(A) op(A)^T + beta C on the named
    triangle only; the other triangle is left as it was."""
    rng = np.random.default_rng(5)
    n, k = 60, 41
    ar, ac = (k, n) if tra == "T" else (n, k)
    A = np.asfortranarray(rng.normal(size=(ar + 2, ac)))
    C = np.asfortranarray(rng.normal(size=(n + 4, n)))
    op = A[:ar].T if tra == "T" else A[:ar]
    full = 2.0 * op @ op.T + 0.25 * C[:n]
    mask = np.triu(np.ones((n, n), bool)) if uplo == "U" else np.tril(np.ones((n, n), bool))
    ref = C.copy(order="F")
    ref[:n][mask] = full[mask]
    _L().call_syrk_cublas(uplo.encode(), tra.encode(), n, k, 2.0, _p(A), ar + 2, 0.25, _p(C), n + 4)
    np.testing.assert_allclose(C, ref, atol=1e-12)


def test_diag_for_gpu_shim_is_the_oracle_pseudo_diagonalisation():
    """diag_for_GPU(fao, vector, nocc, eig, norbs, mpack)
    (matrix/diag_for_GPU.F90:16-234): Fmo, tiny and the ordered sweep."""
    s = oracle_system(*SYSTEMS["water16"])
    r = so.iter_scf(s, itrmax=6)
    f = s.h.copy()
    so.fock2(s, f, r.p, r.p * 0.5)
    c0, e0 = so.eigenvectors_lapack(f.copy(), s.norbs)
    f2 = f + np.random.default_rng(1).normal(scale=1e-3, size=f.shape)
    ref = c0.copy(order="F")
    so.pseudo_diag(f2, ref, s.nclose, e0)
    got = c0.copy(order="F")
    _L().diag_for_gpu_(_p(f2), _p(got), _i(s.nclose), _p(e0), _i(s.norbs), _i(s.mpack))
    np.testing.assert_allclose(got, ref, atol=1e-12)


def test_helect_and_cnvg_shims():
    """helect(n, p, h, f) (integrals/helect.F90) and cnvg(pnew, p, p1, niter, pl)
    (SCF/cnvg.F90; norbs from mb_set_norbs_, as molkst_C gives it to cnvg)."""
    s = oracle_system(*SYSTEMS["propane"])
    p = mixed_density(s)
    f = s.h.copy()
    so.fock2(s, f, p, p * 0.5)
    e = _L().helect_(_i(s.norbs), _p(p), _p(s.h), _p(f))
    assert abs(e - so.helect(s.norbs, p, s.h, f)) < 1e-9 * abs(e)
    rng = np.random.default_rng(2)
    pn = p + rng.normal(scale=1e-3, size=p.shape)
    po = p.copy()
    p1 = p[so.diag_index(s.norbs)] * 0.99
    rn, ro_, r1 = pn.copy(), po.copy(), p1.copy()
    plr = so.cnvg(s.norbs, rn, ro_, r1, 6)
    _L().mb_set_norbs_(_i(s.norbs))
    pl = ctypes.c_double(0.0)
    _L().cnvg_(_p(pn), _p(po), _p(p1), _i(6), ctypes.byref(pl))
    assert pl.value == plr
    assert np.array_equal(pn, rn) and np.array_equal(po, ro_) and np.array_equal(p1, r1)


def test_mozyme_shims_with_registered_arrays():
    """density_for_MOZYME(p, mode, nclose, partp), buildf(f, partf, 0) and
    diagg(fao, nocc, nvir, idiagg, partp, indi) (MOZYME/density_for_MOZYME.F90,
    buildf.F90, diagg.F90) through their gfortran names, after the host has
    registered its MOZYME_C arrays (mb_mz_bind_system_, mb_mz_bind_lmos_,
    mb_mz_bind_controls_): each against the oracle's restatement, bit for bit,
    and the host arrays hold diagg's results afterwards."""
    from mopac_gpu_b200 import workloads
    from oracle import mozyme_oracle as mo
    nat, xyz, _ = workloads.water_box(32)
    s = oracle_system(nat, xyz)
    iorbs = np.ascontiguousarray((s.nlast - s.nfirst + 1).astype(np.int32))
    c1, c2 = mo.cutoffs(len(nat), 9.0)
    mp, nb = mo.layout(iorbs, s.coord, c1, c2)
    h = np.ascontiguousarray(mo.dense_to_blocks(so.unpack(s.h, s.norbs), iorbs, nb, mp))
    w = np.ascontiguousarray(mo.w_stored(iorbs, nb, s.w))
    _, occ = workloads.mozyme_lmos(nat, xyz, radius=4.0, seed=3, per_heavy=4, pad_atoms=2)
    _, vir = workloads.mozyme_lmos(nat, xyz, radius=3.2, seed=4, per_heavy=2, pad_atoms=2)
    occ = [np.ascontiguousarray(x) for x in occ]
    vir = [np.ascontiguousarray(x) for x in vir]
    L = _L()
    coord = np.ascontiguousarray(s.coord.reshape(-1))
    nw = ctypes.c_longlong(w.size)
    assert L.mb_mz_bind_system_(_i(len(nat)), _p(iorbs), _p(coord), _d(c1), _d(c2), _p(h), _p(w),
                                ctypes.byref(nw)) == 0
    p = np.zeros(mp)
    eigs = np.zeros(len(occ[0]) + len(vir[0]))
    cap = 300 * s.norbs
    ll = lambda v: ctypes.byref(ctypes.c_longlong(int(v)))
    assert L.mb_mz_bind_lmos_(_i(len(occ[0])), _p(occ[0]), _p(occ[1]), _p(occ[2]), _p(occ[3]), _p(occ[4]),
                              ll(occ[2].size), ll(occ[4].size), _i(len(vir[0])), _p(vir[0]), _p(vir[1]),
                              _p(vir[2]), _p(vir[3]), _p(vir[4]), ll(vir[2].size), ll(vir[4].size), _p(p),
                              _p(eigs), ll(cap)) == 0
    shift, thresh = ctypes.c_double(0.0), ctypes.c_double(1.0e-13)
    assert L.mb_mz_bind_controls_(ctypes.byref(shift), ctypes.byref(thresh)) == 0
    partp = np.zeros(mp)
    # density_for_MOZYME
    L.density_for_mozyme_(_p(p), _i(0), _i(len(occ[0])), _p(partp))
    p_ref = mo.density(iorbs, nb, tuple(occ), 0, mp)
    assert np.array_equal(p, p_ref)
    # buildf (whole F from the registered p)
    f = np.zeros(mp)
    L.buildf_(_p(f), _p(partp), _i(0))
    f_ref = mo.fock(s.nat, s.coord, iorbs, nb, s.w, p_ref, h)
    assert np.array_equal(f, f_ref)
    # diagg: diagg1 + diagg2 + density, the host arrays updated in place
    o_ref, v_ref = tuple(x.copy() for x in occ), tuple(x.copy() for x in vir)
    st = np.array([10.0, 1.0, 0.0, 0.0])
    nfmo = np.zeros(len(vir[0]), np.int32)
    ifmo = np.zeros(2 * cap, np.int32)
    fmo = np.zeros(cap)
    nij, eigv, eg, _ = mo.diagg1(iorbs, nb, f_ref, p_ref, o_ref, v_ref, 0, st, nfmo, ifmo, fmo, cap)
    mo.diagg2(iorbs, o_ref, v_ref, ifmo, fmo, nij, eg, eigv, 0, [1.0, 0.0, 1e-13, st[3], 50 * np.sqrt(1e-39)],
              np.zeros(2, np.int32))
    p2_ref = mo.density(iorbs, nb, o_ref, 0, mp)
    L.diagg_(_p(f), _i(len(occ[0])), _i(len(vir[0])), _i(0), _p(partp), _i(0))
    for got, ref in zip(occ + vir, o_ref + v_ref):
        assert np.array_equal(got, ref)
    assert np.array_equal(p, p2_ref)
    np.testing.assert_array_equal(eigs[:len(occ[0])], eg)
    np.testing.assert_array_equal(eigs[len(occ[0]):], eigv)
    L.mopac_cuda_destroy_resources()
