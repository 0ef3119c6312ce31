"""Learned initial guess on the GPU against the CPU oracle.

Pairs, frames, descriptors, training targets and the assembly must match the
oracle (integer pair sets exactly, geometry to 1e-10); the BF16 network's
forward pass and gradients match the oracle's BF16 statement within a few
BF16 ulps (outputs 2e-2 relative, gradient norms 3e-2 relative); an SCF
started from a supplied density follows the oracle's iteration by iteration;
and an SCF started from the trained network converges to the standard SCF's
heat (1e-4 kcal/mol) in fewer iterations.
"""
import ctypes

import numpy as np
import pytest

from oracle import guess_oracle as go
from oracle import scf_oracle as so

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.fixture(scope="module")
def cluster():
    from mopac_gpu_b200 import workloads
    nat, xyz = workloads.water_lattice(12, seed=3)
    s = so.make_system(nat, xyz)
    r = so.iter_scf(s)
    return nat, xyz, s, r


def _sorted_pairs(F, S, T):
    return sorted(zip((int(v) for v in T), (int(v) for v in F), (int(v) for v in S)))


def test_pairs_frames_descriptors_match_oracle(cluster):
    from mopac_gpu_b200.guess import PairSet
    nat, xyz, _, _ = cluster
    ps = PairSet(nat, xyz)
    F, S, T = go.pair_list(nat, xyz)
    pf, pss, pt = ps.pf.cpu().numpy(), ps.ps.cpu().numpy(), ps.pt.cpu().numpy()
    assert _sorted_pairs(pf, pss, pt) == _sorted_pairs(F, S, T)
    assert list(np.bincount(T, minlength=5)) == ps.counts
    Xo, Ro = go.features(nat, xyz, pf, pss, pt)
    Xg = ps.feat.cpu().numpy().astype(np.float64)
    Rg = ps.frames.cpu().numpy().reshape(-1, 3, 3).transpose(0, 2, 1)  # columns are axes
    assert np.abs(Rg - Ro).max() < 1e-10
    assert np.abs(Xg - Xo).max() <= 1e-5 * max(1.0, np.abs(Xo).max())


def test_targets_and_assembly_match_oracle(cluster):
    from mopac_gpu_b200.guess import PairSet, GuessModel
    nat, xyz, s, r = cluster
    ps = PairSet(nat, xyz)
    pf, pss, pt = ps.pf.cpu().numpy(), ps.ps.cpu().numpy(), ps.pt.cpu().numpy()
    Ro = ps.frames.cpu().numpy().reshape(-1, 3, 3).transpose(0, 2, 1)
    p_dev = torch.tensor(r.p, dtype=torch.float64, device="cuda")
    y = ps.targets(p_dev.data_ptr()).cpu().numpy().astype(np.float64)
    yo = go.local_blocks(r.p, nat, pf, pss, pt, Ro)
    assert np.abs(y - yo).max() < 1e-6  # float32 storage of the blocks
    # assembly of the (normalised) blocks through an identity-normalised model
    blob = go.init_blob(0)
    model = GuessModel(blob)
    yt = torch.tensor(yo, dtype=torch.float32, device="cuda")
    out = torch.zeros(s.mpack, dtype=torch.float64, device="cuda")
    from mopac_gpu_b200._lib import lib
    rc = lib().mb_guess_assemble_dev(model.handle, ps.n, ps.pf.data_ptr(), ps.ps.data_ptr(), ps.pt.data_ptr(),
                                     ps.frames.data_ptr(), yt.data_ptr(), ps.first.data_ptr(), ps.nor.data_ptr(),
                                     out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    pg = out.cpu().numpy()
    po = go.assemble(nat, pf, pss, pt, Ro, yo.astype(np.float32).astype(np.float64))
    assert np.abs(pg - po).max() < 1e-12
    covered = po != 0
    assert np.abs(pg - r.p)[covered].max() < 1e-6


def _rand_rows(n, seed):
    rng = np.random.default_rng(seed)
    x = go.bf16(rng.normal(size=(n, go.DIN)).astype(np.float32))
    yt = rng.normal(size=(n, go.DOUT)).astype(np.float32)
    return x, yt


def _bits(x):
    return torch.tensor(go.bf16_bits(x).view(np.int16), device="cuda")


@pytest.mark.parametrize("t", [0, 2, 3])
def test_forward_matches_oracle(t):
    from mopac_gpu_b200.guess import GuessModel
    from mopac_gpu_b200._lib import lib
    blob = go.init_blob(5)
    model = GuessModel(blob)
    n = 200  # not a multiple of the 64-row tile
    x, _ = _rand_rows(n, 7)
    xd = _bits(x)
    y = torch.empty((n, go.DOUT), dtype=torch.float32, device="cuda")
    ws = torch.empty(2 * n * go.HID, dtype=torch.int16, device="cuda")
    assert lib().mb_guess_forward_dev(model.handle, t, n, xd.data_ptr(), y.data_ptr(), ws.data_ptr(),
                                      torch.cuda.current_stream().cuda_stream) == 0
    yo, _ = go.forward(go.unpack_blob(blob)[t], x)
    yg = y.cpu().numpy()
    assert np.linalg.norm(yg - yo) <= 2e-2 * np.linalg.norm(yo)
    assert np.abs(yg - yo).max() <= 5e-2 * np.abs(yo).max()


@pytest.mark.parametrize("t", [0, 3])
def test_trainer_gradients_and_adam_match_oracle(t):
    from mopac_gpu_b200.guess import Trainer
    blob = go.init_blob(6)
    n = 256
    x, yt = _rand_rows(n, 8)
    tr = Trainer(blob, n)
    xd = _bits(x)
    ytd = torch.tensor(yt, device="cuda")
    loss = tr.step(t, xd, ytd, 1e-3, update=False, want_loss=True)
    _, grads = tr.get()
    p = go.unpack_blob(blob)[t]
    lo, go_grads, _ = go.loss_and_grads(p, x, yt, int(go.NOUT[t]))
    assert abs(loss - lo) <= 1e-2 * lo
    gg = go.unpack_blob(grads)[t]
    for k in go.TRAINABLE:
        assert np.linalg.norm(gg[k] - go_grads[k]) <= 3e-2 * np.linalg.norm(go_grads[k]), k
    # one Adam step from the same state moves every weight like the oracle's
    tr.step(t, xd, ytd, 1e-3, update=True)
    params, grads2 = tr.get()
    p_or = {k: v.copy() for k, v in go.unpack_blob(blob)[t].items()}
    g2 = go.unpack_blob(grads2)[t]
    m = {k: np.zeros_like(p_or[k]) for k in go.TRAINABLE}
    v = {k: np.zeros_like(p_or[k]) for k in go.TRAINABLE}
    go.adam(p_or, {k: g2[k] for k in go.TRAINABLE}, m, v, 1, 1e-3)
    pg = go.unpack_blob(params)[t]
    for k in go.TRAINABLE:
        assert np.abs(pg[k] - p_or[k]).max() <= 1e-6, k
    tr.close()


def test_training_reduces_loss_on_device():
    from mopac_gpu_b200.guess import Trainer
    blob = go.init_blob(7)
    n = 512
    x, yt = _rand_rows(n, 9)
    tr = Trainer(blob, n)
    xd, ytd = _bits(x), torch.tensor(yt, device="cuda")
    l0 = tr.step(2, xd, ytd, 1e-3, update=False, want_loss=True)
    for _ in range(60):
        tr.step(2, xd, ytd, 1e-3)
    l1 = tr.step(2, xd, ytd, 1e-3, update=False, want_loss=True)
    assert l1 < 0.5 * l0
    tr.close()


def test_scf_from_supplied_density_follows_oracle(cluster):
    from mopac_gpu_b200 import ScfContext
    nat, xyz, s, r = cluster
    rng = np.random.default_rng(3)
    g = r.p + rng.normal(scale=2e-3, size=r.p.shape) * (np.abs(r.p) > 1e-3)
    ro = so.iter_scf(s, p_guess=g)
    ctx = ScfContext(nat, xyz)
    ctx.set_hw(s.h, s.w, s.enuclr)
    ctx.set_guess(g)
    rg = ctx.run(guess=True)
    assert rg.converged and rg.niter == ro.niter
    assert abs(rg.escf - ro.escf) < 1e-6
    assert np.abs(ctx.density() - ro.p).max() < 1e-6
    # a guess run needs a guess
    ctx2 = ScfContext(nat, xyz)
    ctx2.hcore()
    from mopac_gpu_b200 import LibraryError
    with pytest.raises(LibraryError):
        ctx2.run(guess=True)
    ctx.close()
    ctx2.close()


def test_device_prediction_matches_oracle(cluster):
    from mopac_gpu_b200 import ScfContext
    from mopac_gpu_b200.guess import GuessModel
    nat, xyz, s, _ = cluster
    rng = np.random.default_rng(4)
    blob = go.init_blob(8)
    for tp in go.unpack_blob(blob):   # small, varied outputs
        tp["W4"][:] *= 0.05
        tp["out_mean"][:] = rng.normal(scale=0.1, size=go.DOUT)
        tp["out_std"][:] = 0.05
        tp["in_std"][:] = 2.0
    model = GuessModel(blob)
    ctx = ScfContext(nat, xyz)
    ctx.hcore()
    ctx.learned_guess(model)
    from mopac_gpu_b200._lib import lib
    # the entry point the context uses, into a buffer of our own
    from mopac_gpu_b200.guess import PairSet
    ps = PairSet(nat, xyz)
    out = torch.empty(s.mpack, dtype=torch.float64, device="cuda")
    assert lib().mb_guess_predict_density_dev(model.handle, len(nat), ps.nat.data_ptr(), ps.xyz.data_ptr(),
                                              ps.first.data_ptr(), ps.nor.data_ptr(), ps.norbs, out.data_ptr(),
                                              torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    pg = out.cpu().numpy()
    po = go.predict_density(blob, nat, xyz)
    assert np.abs(pg - po).max() <= 2e-2 * np.abs(po).max()
    r = ctx.run(guess=True)  # converges from a poor guess; the SCF decides
    assert r.converged
    ctx.close()


def test_purification_matches_oracle(cluster):
    from mopac_gpu_b200._lib import lib
    nat, xyz, s, r = cluster
    rng = np.random.default_rng(7)
    g = r.p + rng.normal(scale=3e-3, size=r.p.shape) * (np.abs(r.p) > 1e-3)
    for steps in (0, 1, 2):
        p = torch.tensor(g, dtype=torch.float64, device="cuda")
        ws = torch.empty(int(lib().mb_guess_purify_ws_bytes(s.norbs)), dtype=torch.uint8, device="cuda")
        assert lib().mb_guess_purify_dev(s.norbs, p.data_ptr(), steps, ws.data_ptr(),
                                         torch.cuda.current_stream().cuda_stream) == 0
        torch.cuda.synchronize()
        po = go.purify(g, s.norbs, steps) if steps else g
        assert np.abs(p.cpu().numpy() - po).max() < 1e-10, steps


def test_split_purification_matches_oracle_to_the_split_gemm_bound(cluster):
    """mb_ctx_guess's purification: the same McWeeny steps with the products
    as three-product BF16 splits (about 1e-5 of |A||B| per element)."""
    from mopac_gpu_b200._lib import lib
    nat, xyz, s, r = cluster
    rng = np.random.default_rng(7)
    g = r.p + rng.normal(scale=3e-3, size=r.p.shape) * (np.abs(r.p) > 1e-3)
    n = s.norbs
    tc = torch.empty(int(lib().mb_gemm_split_ws_bytes(n, n, n)) + 1024, dtype=torch.uint8, device="cuda")
    tc_ptr = (tc.data_ptr() + 1023) & ~1023
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    for steps in (0, 1, 2):
        p = torch.tensor(g, dtype=torch.float64, device="cuda")
        ws = torch.empty(int(lib().mb_guess_purify_ws_bytes(n)), dtype=torch.uint8, device="cuda")
        assert lib().mb_guess_purify_split_dev(n, p.data_ptr(), steps, ws.data_ptr(), tc_ptr,
                                               int(lib().mb_gemm_split_ws_bytes(n, n, n)), err.data_ptr(),
                                               torch.cuda.current_stream().cuda_stream) == 0
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        po = go.purify(g, n, steps) if steps else g
        dev = np.abs(p.cpu().numpy() - po).max()
        assert dev < (1e-12 if steps == 0 else 1e-4), (steps, dev)


def test_trained_network_cuts_iterations_and_keeps_the_heat():
    from mopac_gpu_b200.guess import GuessModel, evaluate
    if not GuessModel.available():
        pytest.skip("no trained parameter blob in mopac_gpu_b200/data")
    model = GuessModel()
    ev = evaluate(model, n_clusters=6, nmin=32, nmax=64, seed=4242)
    assert ev.max_dhf < 1e-4
    assert ev.n_fallback == 0
    assert ev.niter_learned < ev.niter_std
