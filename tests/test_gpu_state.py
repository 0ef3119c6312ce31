"""mopac_state save/load and DENOUT -> OLDENS on the GPU context: a saved
converged state restarts the SCF in a few iterations with the same heat
(1e-4 kcal/mol), like MOPAC's OLDENS; the oracle's SCF from the same density
takes the same iterations."""
import numpy as np
import pytest

from oracle import scf_oracle as so

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_state_round_trip_restarts_the_scf(tmp_path):
    from mopac_gpu_b200 import LibraryError, ScfContext, workloads
    from mopac_gpu_b200.state import MopacState, denout, load_state, oldens, save_state
    nat, xyz = workloads.water_lattice(16)
    s = so.make_system(nat, xyz)
    ctx = ScfContext(nat, xyz)
    ctx.set_hw(s.h, s.w, s.enuclr)
    r0 = ctx.run()
    st = save_state(ctx)
    assert st.mpack == s.mpack and st.uhf == 0
    np.testing.assert_array_equal(st.pa * 2.0, ctx.density())
    # mopac_load: restart from the state
    ctx2 = ScfContext(nat, xyz)
    ctx2.set_hw(s.h, s.w, s.enuclr)
    load_state(ctx2, st)
    r1 = ctx2.run(guess=True)
    ro = so.iter_scf(s, p_guess=st.pa * 2.0)
    assert r1.converged and abs(r1.escf - r0.escf) < 1e-4
    assert r1.niter == ro.niter and r1.niter < r0.niter
    # DENOUT -> OLDENS through a file, both formats
    for formatted in (False, True):
        f = tmp_path / f"w16_{int(formatted)}.den"
        denout(ctx, f, formatted)
        ctx3 = ScfContext(nat, xyz)
        ctx3.set_hw(s.h, s.w, s.enuclr)
        assert oldens(ctx3, f) == formatted
        r3 = ctx3.run(guess=True)
        assert r3.niter == r1.niter and abs(r3.escf - r1.escf) < 1e-9
        ctx3.close()
    with pytest.raises(LibraryError, match="incompatible"):
        load_state(ctx2, MopacState(st.mpack - 1, 0, st.pa[:-1], None))
    ctx.close()
    ctx2.close()
