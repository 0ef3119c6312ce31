"""Pin the CPU oracle to the reference's own golden outputs.

The values in tests/golden/reference_values.json were extracted from the
reference's test files by tests/golden/make_golden.py (sources listed there).
They are printed to 5 (eigenvalues, heats) or 6 (charges) decimals.
"""
import json
import os

import numpy as np
import pytest

from oracle import scf_oracle as so

G = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_values.json")))


def _run(case, **kw):
    s = so.make_system(case["nat"], case["xyz"])
    return s, so.iter_scf(s, **kw)


@pytest.mark.parametrize("name", ["co2_1scf", "propane"])
def test_eigenvalues_match_reference_output(name):
    case = G[name]
    s, r = _run(case)
    assert r.converged
    # printed with 5 decimals: allow one unit in the last place
    np.testing.assert_allclose(r.eigs, case["eigs"], atol=1.01e-5, rtol=0)


@pytest.mark.parametrize("name", ["co2_1scf", "propane", "h2o_api"])
def test_charges_match_reference_output(name):
    case = G[name]
    s, r = _run(case)
    q = so.mulliken_charges(s, r.p)
    # the API test's own tolerance is 1e-3 (mopac_api_test.F90:2211-2216); the
    # keyword outputs match to their printed 6 decimals at default SCFCRT
    tol = 1e-5 if name != "h2o_api" else 1e-4
    np.testing.assert_allclose(q, case["charges"], atol=tol, rtol=0)


def test_h2o_heat_matches_reference_exactly():
    case = G["h2o_api"]
    s, r = _run(case)
    assert abs(so.heat_of_formation(s, r) - case["heat"]) < 1.0e-5


@pytest.mark.parametrize("name", ["co2_1scf", "propane"])
def test_keyword_output_heats_within_the_reference_suites_bound(name):
    """The keyword outputs (tests/keywords/1SCF.out, VECTORS.out) were written
    by MOPAC2016 21.298M (2021, their banner); the source is 23.1.2
    (CITATION.cff).  The reference's own harness checks these stored heats
    against the current build with HOF_ERROR = 0.01 kcal/mol
    (tests/CMakeLists.txt:18, compare_output.py:244) and warns above 1e-4
    (compare_output.py:29, :245).  The oracle lands 3.1e-4 (CO2) and 7.9e-4
    (propane) from them, inside that bound, while the ionisation potentials of
    the same files match to 1e-7 eV and the current-source API heat (water,
    above) to 4e-6; the bar here is the reference suite's own 0.01, with the
    measured residual pinned below 1e-3 so a regression shows."""
    case = G[name]
    s, r = _run(case)
    d = abs(so.heat_of_formation(s, r) - case["heat"])
    assert d < 1.0e-2
    assert d < 1.0e-3


def test_tight_convergence_is_stable():
    case = G["propane"]
    s, r1 = _run(case)
    s, r2 = _run(case, scfcrt=1e-9)
    assert abs(r1.escf - r2.escf) < 1e-4
    np.testing.assert_allclose(r1.eigs, r2.eigs, atol=2e-5)


def test_w_layout_size_matches_reference_sizing():
    # moldat.F90:290-293 sizing for sp elements
    from math import comb
    for n4, n1 in [(1, 2), (16, 32), (3, 8)]:
        nat = [8] * n4 + [1] * n1
        n2 = so.lib().orc_n2elec(len(nat), np.array(nat, np.int32))
        assert n2 + 10 == 100 * comb(n4, 2) + 100 * n4 + n1 + 10 * n4 * n1 + comb(n1, 2) + 10
