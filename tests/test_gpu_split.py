"""Split-precision tensor-core GEMMs (tcgen05, three BF16 products) and the
SCF's precision switch with its FP64 finish.

Tolerance of the split products: |C - C_fp64| <= 1e-4 * (|A| |B|) element by
element (three BF16 products leave ~2^-16 relative per product; FP32
accumulation adds ~k 2^-24 in the worst case).

The SCF with the switch on takes a different path from the FP64 one; iter's
own convergence test stops 1e-5..1e-4 away from the self-consistent density,
so the split SCF finishes in FP64 (mb_scf_opts.finish_dp, 1e-7 by default
with precision = 1) until the density stops moving, and is held to the
self-consistent point of the FP64 oracle: heat 1e-4 kcal/mol, density 1e-6,
orbital energies 1e-5 eV.
"""
import ctypes

import numpy as np
import pytest

from oracle import scf_oracle as so
from tests.helpers import oracle_system, small_systems

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
SYSTEMS = small_systems()


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _dev_colmajor(a):
    return torch.from_numpy(np.ascontiguousarray(np.asfortranarray(a).ravel(order="F"))).cuda()


def _gemm_split(ta, tb, a, b, alpha=1.0, beta=0.0, c0=None):
    from mopac_gpu_b200._lib import check, lib
    opa = a.T if ta == "T" else a
    opb = b.T if tb == "T" else b
    m, k = opa.shape
    n = opb.shape[1]
    da, db = _dev_colmajor(a), _dev_colmajor(b)
    c = c0 if c0 is not None else np.zeros((m, n))
    dc = _dev_colmajor(c)
    nb = int(lib().mb_gemm_split_ws_bytes(m, n, k))
    buf = torch.empty(nb + 1024, dtype=torch.uint8, device="cuda")
    ws = ctypes.c_void_p((buf.data_ptr() + 1023) & ~1023)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    check(lib().mb_gemm_split_ws(ta.encode(), tb.encode(), m, n, k, alpha, ctypes.c_void_p(da.data_ptr()),
                                 a.shape[0], ctypes.c_void_p(db.data_ptr()), b.shape[0], beta,
                                 ctypes.c_void_p(dc.data_ptr()), m, ws, nb, ctypes.c_void_p(err.data_ptr()), s))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return dc.cpu().numpy().reshape(n, m).T, opa, opb


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
@pytest.mark.parametrize("m,n,k", [(128, 128, 64), (200, 77, 130), (1, 300, 5), (513, 257, 1000)])
def test_gemm_split_matches_fp64(ta, tb, m, n, k):
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    a = rng.normal(size=(k, m) if ta == "T" else (m, k))
    b = rng.normal(size=(n, k) if tb == "T" else (k, n))
    c, opa, opb = _gemm_split(ta, tb, a, b, alpha=0.75)
    ref = 0.75 * opa @ opb
    bound = 1e-4 * 0.75 * (np.abs(opa) @ np.abs(opb)) + 1e-12
    assert np.all(np.abs(c - ref) <= bound)


def test_gemm_split_beta_accumulates():
    rng = np.random.default_rng(11)
    a, b, c0 = rng.normal(size=(150, 90)), rng.normal(size=(90, 140)), rng.normal(size=(150, 140))
    c, opa, opb = _gemm_split("N", "N", a, b, alpha=2.0, beta=-0.5, c0=c0)
    ref = 2.0 * a @ b - 0.5 * c0
    assert np.all(np.abs(c - ref) <= 2e-4 * (np.abs(a) @ np.abs(b)) + 1e-12)


@pytest.mark.parametrize("n,nocc", [(96, 64), (300, 131), (1000, 700), (3072, 2048)])
def test_density_split_matches_fp64(n, nocc):
    from mopac_gpu_b200 import kernels
    rng = np.random.default_rng(n)
    q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    c = torch.from_numpy(np.ascontiguousarray(q)).cuda()          # row-major storage of C
    cc = c.t().contiguous().t()                                    # column-major view
    p64 = kernels.density(cc, nocc).cpu().numpy()
    psp = kernels.density_split(cc, nocc).cpu().numpy()
    co = q[:, :nocc]
    ref = so.pack(2.0 * co @ co.T)
    np.testing.assert_allclose(p64, ref, atol=1e-12)
    bound = so.pack(1e-4 * 2.0 * np.abs(co) @ np.abs(co).T) + 1e-12
    assert np.all(np.abs(psp - ref) <= bound)


def test_matmul_split_wrapper():
    from mopac_gpu_b200 import kernels
    rng = np.random.default_rng(2)
    a, b = rng.normal(size=(64, 33)), rng.normal(size=(33, 250))
    c = kernels.matmul_split(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()).cpu().numpy()
    assert np.all(np.abs(c - a @ b) <= 1e-4 * (np.abs(a) @ np.abs(b)) + 1e-12)


def _fixed_point(s):
    """The oracle's self-consistent point: plain iter run to 1e-11 in P."""
    return so.iter_scf(s, scfcrt=1.0e-12, finish_dp=1.0e-11, finish_max=200)


@pytest.mark.parametrize("name", ["water16", "propane", "heptane", "co2_1scf"])
@pytest.mark.parametrize("pseudo,pulay", [(False, False), (True, False), (True, True)])
def test_split_precision_scf_lands_on_fp64_oracle(name, pseudo, pulay):
    from mopac_gpu_b200 import ScfContext
    nat, xyz = SYSTEMS[name]
    s = oracle_system(nat, xyz)
    ref = _fixed_point(s)
    ctx = ScfContext(nat, xyz)
    ctx.set_hw(s.h, s.w, s.enuclr)
    r = ctx.run(pseudo=pseudo, pulay=pulay, precision=1, switch_pl=1e-4)
    p = ctx.density()
    _, e = ctx.vectors()
    ctx.close()
    assert r.converged and r.n_split > 0 and r.dp <= 1e-7
    print(f"{name} pseudo={pseudo} pulay={pulay}: dHf {r.escf - ref.escf:.2e} kcal/mol, "
          f"max|dP| {np.abs(p - ref.p).max():.2e}, max|de| {np.abs(e - ref.eigs).max():.2e} eV, "
          f"split iterations {r.n_split}, finish {r.n_finish} of {r.niter}")
    assert abs(r.escf - ref.escf) < 1e-4
    assert np.abs(p - ref.p).max() < 1e-6
    assert np.abs(e - ref.eigs).max() < 1e-5


def test_split_scf_matches_the_oracle_running_the_same_finish():
    """Same algorithm on both sides (pseudo-diagonalisation, Pulay, finish):
    the GPU's split SCF and the oracle's FP64 one end within 1e-6."""
    from mopac_gpu_b200 import ScfContext, workloads
    nat, xyz, _ = workloads.water_box(32)
    s = oracle_system(nat, xyz)
    ref = so.iter_scf(s, pseudo=True, pulay_on=True, finish_dp=1.0e-7)
    ctx = ScfContext(nat, xyz)
    ctx.set_hw(s.h, s.w, s.enuclr)
    r = ctx.run(pseudo=True, pulay=True, precision=1)
    p = ctx.density()
    c, e = ctx.vectors()
    fk = ctx.fock()
    ctx.close()
    assert r.converged and ref.converged
    assert abs(r.escf - ref.escf) < 1e-4
    assert np.abs(p - ref.p).max() < 1e-6
    assert np.abs(e - ref.eigs).max() < 1e-5
    # the exit diagonalisation ran as the occupied and virtual blocks: its
    # vectors are eigenvectors of the (perturbed) F as tightly as the whole
    # eigensolve's, and orthonormal
    fp = so.unpack(fk, s.norbs)
    fp[np.diag_indices(s.norbs)] += np.arange(1, s.norbs + 1) * 1.0e-10
    print(f"exit split {r.exit_split}, ||B||_F {r.exit_coupling:.2e} eV, "
          f"max|F C - C e| {np.abs(fp @ c - c * e).max():.2e}")
    assert r.exit_split and 0.0 <= r.exit_coupling < 1e-3
    assert np.abs(fp @ c - c * e).max() < 1e-9
    assert np.abs(c.T @ c - np.eye(s.norbs)).max() < 1e-10


def test_finish_off_keeps_iter_semantics():
    """finish_dp = 0 on the FP64 path is iter unchanged: same iterations and
    density as the oracle without the finish."""
    from mopac_gpu_b200 import ScfContext
    nat, xyz = SYSTEMS["water16"]
    s = oracle_system(nat, xyz)
    ref = so.iter_scf(s, pseudo=True, pulay_on=True)
    ctx = ScfContext(nat, xyz)
    ctx.set_hw(s.h, s.w, s.enuclr)
    r = ctx.run(pseudo=True, pulay=True, precision=0, finish_dp=0.0)
    p = ctx.density()
    ctx.close()
    assert r.n_finish == 0 and r.dp == -1.0 and r.niter == ref.niter
    assert np.abs(p - ref.p).max() < 1e-7
