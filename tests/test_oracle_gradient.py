"""The oracle's dcart (forces/dcart.F90, a molecule, RHF) checked against
itself and against the SCF energy: the pair energies behind it give, by a
central difference, the derivative of the converged SCF energy (the energy is
variational in P, so only the pairs' geometry enters); the reference's own
half-step scheme (atom jj moved chnge/2 along all axes before each move of
atom ii) carries an O(chnge) cross term of the pairs' force constants, so its
result sits within 0.05 kcal/mol/A of that derivative (0.022 for propane's
C-H pairs); and every gradient sums to zero over the
atoms."""
import json
import os

import numpy as np
import pytest

from oracle import scf_oracle as so

G = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_values.json")))


def _system(name):
    v = G[name]
    s = so.make_system(np.array(v["nat"], np.int32), np.array(v["xyz"], float))
    return s, so.iter_scf(s, scfcrt=1e-12)


def _central(s, p, h=1e-4):
    P = so.unpack(p, s.norbs)
    g = np.zeros((s.numat, 3))
    for ii in range(s.numat):
        for jj in range(ii):
            idx = np.concatenate([np.arange(s.nfirst[jj] - 1, s.nlast[jj]), np.arange(s.nfirst[ii] - 1, s.nlast[ii])])
            pl = so.pack(P[np.ix_(idx, idx)])
            for k in range(3):
                xp, xm = s.coord[ii].copy(), s.coord[ii].copy()
                xp[k] += h
                xm[k] -= h
                d = (so._pair_energy(s.nat[[jj, ii]], s.coord[jj], xp, pl, 0.5 * pl) -
                     so._pair_energy(s.nat[[jj, ii]], s.coord[jj], xm, pl, 0.5 * pl)) / (2 * h) * so.FPC9
                g[ii, k] += d
                g[jj, k] -= d
    return g


def _numeric(s, a, k, h=1e-4):
    c = s.coord.copy()
    c[a, k] += h
    ep = so.iter_scf(so.make_system(s.nat, c), scfcrt=1e-12).escf
    c[a, k] -= 2 * h
    em = so.iter_scf(so.make_system(s.nat, c), scfcrt=1e-12).escf
    return (ep - em) / (2 * h)


@pytest.mark.parametrize("name", ["propane", "co2_1scf", "h2o_api"])
def test_dcart_against_the_scf_energy(name):
    s, r = _system(name)
    g = so.dcart(s, r.p)
    c = _central(s, r.p)
    assert np.abs(g.sum(axis=0)).max() < 1e-10
    assert np.abs(c.sum(axis=0)).max() < 1e-10
    assert np.abs(g - c).max() < 0.05
    for a, k in [(0, 0), (1, 2), (s.numat - 1, 1)]:
        assert abs(_numeric(s, a, k) - c[a, k]) < 1e-5
