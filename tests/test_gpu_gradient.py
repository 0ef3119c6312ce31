"""dcart on the GPU (mb_ctx_gradient / mb_dcart_dev) against the oracle's
restatement on the same converged density: every pair energy of dhc's form
at the reference's displaced geometries, summed in dcart's order.  The pair
energies agree to about 1e-13 eV; dcart divides their differences by 1e-4 A,
so the bar is 1e-5 kcal/mol/A.  On the (H2O)512 box the check is
size-independent: the gradient sums to zero over the atoms."""
import json
import os

import numpy as np
import pytest

from oracle import scf_oracle as so

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

G = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_values.json")))


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mopac_gpu_b200 import build
    build.build()


def _cases():
    from mopac_gpu_b200 import workloads as wl
    out = {k: (np.array(G[k]["nat"], np.int32), np.array(G[k]["xyz"], float)) for k in ("propane", "co2_1scf")}
    out["water64"] = wl.water_lattice(64)
    out["heptane"] = wl.alkane(7, np.random.default_rng(5))
    return out


@pytest.mark.parametrize("name", ["propane", "co2_1scf", "water64", "heptane"])
def test_gradient_matches_the_oracle(name):
    from mopac_gpu_b200.scf import ScfContext
    nat, xyz = _cases()[name]
    ctx = ScfContext(nat, xyz)
    ctx.hcore()
    ctx.run()
    g = ctx.gradient()
    ref = so.dcart(so.make_system(nat, xyz), ctx.density())
    assert np.abs(g - ref).max() < 1e-5, np.abs(g - ref).max()
    ctx.close()


def test_gradient_of_the_water_box_sums_to_zero():
    from mopac_gpu_b200 import workloads as wl
    from mopac_gpu_b200.scf import ScfContext
    nat, xyz, _ = wl.water_box(512)
    ctx = ScfContext(nat, xyz)
    ctx.hcore()
    ctx.run(pseudo=True)
    g = ctx.gradient()
    assert np.isfinite(g).all()
    assert np.abs(g.sum(axis=0)).max() < 1e-8 * max(1.0, np.abs(g).max())
    ctx.close()
