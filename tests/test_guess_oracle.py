"""CPU checks of the learned-guess oracle: frames, descriptors, block round
trips, the BF16 rounding, and the network's gradients against finite
differences.  These pin the oracle that the GPU kernels are compared with."""
import numpy as np
import pytest

from oracle import guess_oracle as go
from oracle import scf_oracle as so


@pytest.fixture(scope="module")
def cluster():
    from mopac_gpu_b200 import workloads
    nat, xyz = workloads.water_lattice(10, seed=3)
    s = so.make_system(nat, xyz)
    r = so.iter_scf(s)
    return nat, xyz, s, r


def test_pair_list_types_and_order(cluster):
    nat, xyz, _, _ = cluster
    F, S, T = go.pair_list(nat, xyz)
    assert (np.diff(T) >= 0).all()
    for f, s, t in zip(F, S, T):
        if t in (0, 1):
            assert f == s
        elif t == 3:
            assert nat[f] != 1 and nat[s] == 1
        else:
            assert f > s
        assert np.linalg.norm(xyz[f] - xyz[s]) < go.RPAIR
    # every atom has its own block
    assert np.sum(T <= 1) == len(nat)


def test_frames_orthonormal(cluster):
    nat, xyz, _, _ = cluster
    F, S, T = go.pair_list(nat, xyz)
    for f, s in zip(F[::7], S[::7]):
        R = go.frame(int(f), int(s), xyz)
        assert np.allclose(R.T @ R, np.eye(3), atol=1e-12)
        assert np.linalg.det(R) > 0


def test_blocks_round_trip_through_frames(cluster):
    nat, xyz, s, r = cluster
    F, S, T = go.pair_list(nat, xyz)
    _, Rs = go.features(nat, xyz, F, S, T)
    Y = go.local_blocks(r.p, nat, F, S, T, Rs)
    P2 = go.assemble(nat, F, S, T, Rs, Y)
    P, Pm = so.unpack(r.p, s.norbs), so.unpack(P2, s.norbs)
    covered = Pm != 0
    assert np.abs(P - Pm)[covered].max() < 1e-13
    # pairs beyond the cutoff are small: dropping them is a guess error only
    assert np.abs(P[~covered]).max() < 5e-3


def test_descriptors_and_targets_rotation_invariant(cluster):
    nat, xyz, s, r = cluster
    from mopac_gpu_b200 import workloads
    F, S, T = go.pair_list(nat, xyz)
    X, Rs = go.features(nat, xyz, F, S, T)
    Q = workloads._rand_rotation(np.random.default_rng(9))
    xyz2 = xyz @ Q.T + np.array([1.3, -0.4, 2.0])
    X2, Rs2 = go.features(nat, xyz2, F, S, T)
    assert np.abs(X - X2).max() < 1e-10
    r2 = so.iter_scf(so.make_system(nat, xyz2))
    Y = go.local_blocks(r.p, nat, F, S, T, Rs)
    Y2 = go.local_blocks(r2.p, nat, F, S, T, Rs2)
    assert np.abs(Y - Y2).max() < 1e-3  # SCF convergence noise only


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-3], np.float32)
    b = go.bf16(x)
    assert b[0] == 1.0
    assert b[1] == 1.0            # tie -> even
    assert b[2] == 1.0 + 2 ** -7  # above the tie -> up
    assert b[3] == -2.5
    assert abs(b[4] - 3.0e-3) < 3.0e-3 * 2 ** -8
    assert (go.from_bf16_bits(go.bf16_bits(x)) == b).all()


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    p = go.unpack_blob(go.init_blob(1).astype(np.float64))[2]
    x = rng.normal(size=(7, go.DIN))
    yt = rng.normal(size=(7, go.DOUT))
    _, g, _ = go.loss_and_grads(p, x, yt, 16, exact=True)
    for k, idx in (("W1", (3, 100)), ("b1", (9,)), ("b2", (5,)), ("W3", (7, 9)), ("W4", (2, 11)), ("b4", (1,))):
        e = 1e-6
        old = p[k][idx]
        p[k][idx] = old + e
        lp, _, _ = go.loss_and_grads(p, x, yt, 16, exact=True)
        p[k][idx] = old - e
        lm, _, _ = go.loss_and_grads(p, x, yt, 16, exact=True)
        p[k][idx] = old
        fd = (lp - lm) / (2 * e)
        assert abs(g[k][idx] - fd) <= 1e-6 * max(1.0, abs(fd)), (k, g[k][idx], fd)


def test_bf16_gradients_close_to_exact():
    rng = np.random.default_rng(1)
    blob = go.init_blob(2)
    p32 = go.unpack_blob(blob)[3]
    p64 = go.unpack_blob(blob.astype(np.float64))[3]
    x = go.bf16(rng.normal(size=(64, go.DIN)).astype(np.float32))
    yt = rng.normal(size=(64, go.DOUT)).astype(np.float32)
    _, g, _ = go.loss_and_grads(p32, x, yt, 4)
    _, ge, _ = go.loss_and_grads(p64, x.astype(np.float64), yt.astype(np.float64), 4, exact=True)
    for k in go.TRAINABLE:
        assert np.linalg.norm(g[k] - ge[k]) <= 3e-2 * np.linalg.norm(ge[k]), k


def test_adam_decreases_loss():
    rng = np.random.default_rng(2)
    p = go.unpack_blob(go.init_blob(3))[1]
    x = go.bf16(rng.normal(size=(128, go.DIN)).astype(np.float32))
    yt = rng.normal(size=(128, go.DOUT)).astype(np.float32)
    m = {k: np.zeros_like(p[k]) for k in go.TRAINABLE}
    v = {k: np.zeros_like(p[k]) for k in go.TRAINABLE}
    l0, g, _ = go.loss_and_grads(p, x, yt, 1)
    for step in range(1, 21):
        _, g, _ = go.loss_and_grads(p, x, yt, 1)
        go.adam(p, g, m, v, step, 1e-3)
    l1, _, _ = go.loss_and_grads(p, x, yt, 1)
    assert l1 < 0.5 * l0


def test_oracle_scf_from_converged_density_is_short(cluster):
    nat, xyz, s, r = cluster
    r2 = so.iter_scf(s, p_guess=r.p)
    assert r2.converged and abs(r2.escf - r.escf) < 1e-4
    assert r2.niter <= 6 < r.niter


def test_mcweeny_purification_moves_towards_idempotent(cluster):
    nat, xyz, s, r = cluster
    rng = np.random.default_rng(6)
    g = r.p + rng.normal(scale=3e-3, size=r.p.shape) * (np.abs(r.p) > 1e-3)
    n = s.norbs

    def idem(p):
        D = so.unpack(p, n) / 2
        return np.linalg.norm(D @ D - D)
    pp = go.purify(g, n, 1)
    assert idem(pp) < 0.2 * idem(g)
    assert abs(so.unpack(pp, n).trace() - 2 * s.nclose) < 0.05
    assert np.array_equal(go.purify(g, n, 0), so.pack(so.unpack(g, n)))


def test_trained_network_guess_shortens_the_oracle_scf():
    """The committed lattice network, purified once, seeds the oracle's iter:
    same heat (1e-4 kcal/mol), fewer iterations than the diagonal guess."""
    import os
    from mopac_gpu_b200 import workloads
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "mopac_gpu_b200", "data",
                        "guess_pm7_water.npy")
    if not os.path.exists(path):
        pytest.skip("no trained blob")
    blob = np.load(path)
    nat, xyz = workloads.water_lattice(16)
    s = so.make_system(nat, xyz)
    r0 = so.iter_scf(s)
    g = go.purify(go.predict_density(blob, nat, xyz), s.norbs, 1)
    r1 = so.iter_scf(s, p_guess=g)
    assert r1.converged and abs(r1.escf - r0.escf) < 1e-4
    assert r1.niter < r0.niter
