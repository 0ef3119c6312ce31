"""The SCF's FP64 finish and the fixed-point certificate, on the CPU oracle.

iter's convergence test (SCF/iter.F90:675-690: max|dP_ii| < 0.05 sqrt(scfcrt)
and |dE| < scfcrt) stops 1e-5..1e-4 away from the self-consistent density,
so two SCFs that take different paths (split precision, pseudo-diagonalisation,
Pulay) agree with each other, and with the oracle, only to that level.  The
finish (``finish_dp``) carries the SCF on to the self-consistent point; these
tests hold the oracle's own finish to the bar the device SCF is held to
(P within 1e-6, orbital energies within 1e-5 eV, heat within 1e-4 kcal/mol of
the fixed point) and check the certificate the (H2O)512 test relies on.
"""
import numpy as np
import pytest

from mopac_gpu_b200 import workloads as wl
from oracle import scf_oracle as so
from tests.helpers import oracle_system, small_systems


def _fixed_point(s):
    """The self-consistent point: plain iter run to 1e-11 in P."""
    return so.iter_scf(s, scfcrt=1.0e-12, finish_dp=1.0e-11, finish_max=200)


def test_c_rotation_sweep_is_the_python_sweep_bit_for_bit():
    rng = np.random.default_rng(3)
    n, nocc = 90, 50
    c = np.asfortranarray(np.linalg.qr(rng.normal(size=(n, n)))[0])
    fmo = rng.normal(size=(n - nocc, nocc)) * 0.1
    eig = np.sort(rng.normal(size=n)) * 5.0
    for bigeps, tiny in ((1.5e-7, None), (0.0, 0.0), (1.5e-7, 0.02)):
        a, b = c.copy(order="F"), c.copy(order="F")
        na = so.rotation_sweep(a, fmo, eig, nocc, bigeps=bigeps, tiny=tiny)
        nb = so.rotation_sweep_py(b, fmo, eig, nocc, bigeps=bigeps, tiny=tiny)
        assert na == nb and na > 0
        assert np.array_equal(a, b)


def test_iter_stops_inside_its_criterion_not_at_the_fixed_point():
    nat, xyz, _ = wl.water_box(16)
    s = oracle_system(nat, xyz)
    ref = _fixed_point(s)
    std = so.iter_scf(s, pseudo=True, pulay_on=True)
    assert std.n_finish == 0
    assert np.abs(std.p - ref.p).max() > 1e-6   # why the finish exists


@pytest.mark.parametrize("name", ["water16", "propane", "heptane", "box16"])
@pytest.mark.parametrize("mode", [dict(pseudo=True, pulay_on=True), dict(pseudo=True), dict(pseudo=False)])
def test_finish_lands_on_the_fixed_point(name, mode):
    if name.startswith("box"):
        nat, xyz, _ = wl.water_box(int(name[3:]))
    else:
        nat, xyz = small_systems()[name]
    s = oracle_system(nat, xyz)
    ref = _fixed_point(s)
    r = so.iter_scf(s, finish_dp=1.0e-7, **mode)
    assert r.converged and r.n_finish < 40
    assert abs(r.escf - ref.escf) < 1e-6
    assert np.abs(r.p - ref.p).max() < 1e-6
    assert np.abs(r.eigs - ref.eigs).max() < 1e-5


def test_certificate_estimates_the_distance_to_the_fixed_point():
    nat, xyz, _ = wl.water_box(32)
    s = oracle_system(nat, xyz)
    ref = _fixed_point(s)
    for fd in (0.0, 1.0e-7):
        r = so.iter_scf(s, pseudo=True, pulay_on=True, finish_dp=fd)
        err = np.abs(r.p - ref.p).max()
        cert = so.fixed_point_certificate(s, r.p)
        assert 0.3 < cert["rho"] < 0.9
        assert err <= 1.1 * cert["bound"] and cert["bound"] <= 2.0 * err
        # orbital energies of F(p) are what the exit diagonalisation returns
        np.testing.assert_allclose(cert["eigs"], r.eigs, atol=1e-12)
        assert abs(cert["heat_at_p"] - r.escf) < 1e-9


def test_split_exit_diagonalisation_matches_the_whole_eigensolve():
    """After the finish, the exit diagonalisation solved as the occupied and
    virtual blocks of C^T F C (plus the first-order rotation of the
    remaining coupling) gives the whole eigensolve's eigenvalues and vectors
    that satisfy F C = C e as tightly as it does."""
    nat, xyz, _ = wl.water_box(32)
    s = oracle_system(nat, xyz)
    cap = {}
    orig = so.pseudo_diag

    def keep(f, c, nocc, eig, **kw):
        r = orig(f, c, nocc, eig, **kw)
        cap["c"] = c.copy(order="F")
        cap["f"] = f.copy()
        return r

    so.pseudo_diag = keep
    try:
        r = so.iter_scf(s, pseudo=True, pulay_on=True, finish_dp=1.0e-7, shift_kw=0.0)
    finally:
        so.pseudo_diag = orig
    assert r.converged and r.n_finish > 0
    # F of the last iteration is the exit's F (iter.F90 label 600)
    f = s.h.copy()
    so.fock2(s, f, r.p, r.p * 0.5)
    fk = f.copy()
    c, e, bnorm = so.exit_block_diag(fk, cap["c"], s.nclose)
    assert c is not None and bnorm < 1e-3
    np.testing.assert_allclose(e, r.eigs, rtol=0, atol=1e-10)
    fp = so.unpack(fk, s.norbs)
    assert np.abs(fp @ c - c * e).max() < 1e-9
    assert np.abs(c.T @ c - np.eye(s.norbs)).max() < 1e-10
    # the same occupied subspace as the whole eigensolve's
    np.testing.assert_allclose(so.density(c, s.nclose), so.density(r.c, s.nclose), atol=1e-9)
    # a coupling above the bound is declined
    c2, e2, _ = so.exit_block_diag(f.copy(), np.asfortranarray(np.eye(s.norbs)), s.nclose)
    assert c2 is None and e2 is None
