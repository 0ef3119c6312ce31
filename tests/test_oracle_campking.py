"""The Camp-King restatement (oracle/campking_oracle.py) and iter's use of it:
spline and Gram-Schmidt on cases with known answers, then the SCF with CAMP
and with the forced switch-on of all convergers (SCF/iter.F90:351-372)."""
import numpy as np
import pytest

from oracle import scf_oracle as so
from oracle import campking_oracle as ck

# molecules with a positive heat of formation (interp rotates) and one with a
# negative heat (interp analyses the vectors but never rotates them)
ACETYLENE = ([6, 6, 1, 1], [[0, 0, 0.601], [0, 0, -0.601], [0, 0, 1.663], [0, 0, -1.663]])
ETHYLENE = ([6, 6, 1, 1, 1, 1], [[0, 0, 0.667], [0, 0, -0.667], [0, 0.923, 1.238], [0, -0.923, 1.238],
                                 [0, 0.923, -1.238], [0, -0.923, -1.238]])
WATER = ([8, 1, 1], [[0, 0, 0], [0.757, 0.586, 0], [-0.757, 0.586, 0]])


def _system(mol):
    nat, xyz = mol
    return so.make_system(nat, np.array(xyz, dtype=np.float64))


def test_spline_finds_the_minimum_of_a_cubic_through_two_points():
    # f(x) = (x - 0.3)^2 + 1: the Hermite cubic through x = 0 and x = 1 with
    # exact slopes is f itself, whose minimum is at 0.3
    x, f, df = [0.0] * 13, [0.0] * 13, [0.0] * 13
    x[2], f[2], df[2] = 1.0, 1.49, 1.4      # the old point (slot 2)
    x[1], f[1], df[1] = 0.0, 1.09, -0.6     # the current point (slot 1)
    xmin = ck.spline(x, f, df, 10.0, -5.0, 2)
    assert xmin == pytest.approx(0.3, abs=1e-12)
    assert x[1] < x[2]


def test_spline_keeps_the_points_in_x_order():
    x, f, df = [0.0] * 13, [0.0] * 13, [0.0] * 13
    pts = [(0.0, 1.09, -0.6), (1.0, 1.49, 1.4), (0.5, 1.04, 0.4)]
    for i, p in enumerate(pts, start=1):
        x[i], f[i], df[i] = p
    ck.spline(x, f, df, 10.0, -5.0, 3)
    assert x[1:4] == sorted(x[1:4])


def _qr_q(a: np.ndarray) -> np.ndarray:
    q, r = np.linalg.qr(a)
    return q * np.sign(np.diag(r))


def test_schmit_is_gram_schmidt_and_schmib_runs_from_the_last_column():
    rng = np.random.default_rng(5)
    a = rng.normal(size=(9, 9))
    u = np.asfortranarray(a.copy())
    ck.schmit(u, 9)
    assert np.abs(u - _qr_q(a)).max() < 1e-12
    v = np.asfortranarray(a.copy())
    ck.schmib(v, 9)
    assert np.abs(v[:, ::-1] - _qr_q(a[:, ::-1])).max() < 1e-12


def test_schmit_replaces_a_vanishing_column_by_a_unit_vector():
    rng = np.random.default_rng(6)
    a = rng.normal(size=(6, 6))
    a[:, 2] = 0.0
    u = np.asfortranarray(a.copy())
    ck.schmit(u, 6)
    assert np.abs(u.T @ u - np.eye(6)).max() < 1e-12


@pytest.mark.parametrize("mol,rotates", [(ACETYLENE, True), (ETHYLENE, True), (WATER, False)])
def test_camp_king_reaches_the_same_scf(mol, rotates):
    s = _system(mol)
    r0 = so.iter_scf(s)
    r1 = so.iter_scf(s, camp=True)
    assert r0.converged and r1.converged
    assert (r1.n_interp > 0) == rotates
    # both stop inside the 1e-4 kcal/mol criterion of the same fixed point
    assert abs(r1.escf - r0.escf) < 1e-4
    assert np.abs(r1.p - r0.p).max() < 5e-4


@pytest.mark.parametrize("mol", [ACETYLENE, ETHYLENE, WATER])
def test_forced_switch_on_of_all_convergers(mol):
    s = _system(mol)
    r0 = so.iter_scf(s)
    r = so.iter_scf(s, itrmax=14, trace=True)
    assert r.forced_on and r.converged
    assert any(h.get("allcon") for h in r.history)
    assert abs(r.escf - r0.escf) < 1e-4
