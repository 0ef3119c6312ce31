"""dfock2's restatement (oracle/dfock_oracle.py) against the contraction it
stands for: with each pair block of w expanded to (mu nu | lam sig),
F_A(mu, nu) += sum P_B(lam, sig) (mu nu | lam sig), F_B likewise, and
F(mu, lam) -= sum p(nu, sig) (mu nu | lam sig) -- written here with numpy
tensors, independently of the reference's loop and term order."""
import numpy as np
import pytest

from oracle import dfock_oracle as dfo


def _layout(nat):
    first, last, o = [], [], 1
    for z in nat:
        k = 1 if z == 1 else 4
        first.append(o)
        last.append(o + k - 1)
        o += k
    return first, last, o - 1


def _sym_packed(rng, n):
    a = rng.normal(size=(n, n))
    a = a + a.T
    r, c = np.tril_indices(n)
    return a, np.ascontiguousarray(a[r, c])


def _pairs(k):
    """1-based pair index of (a, b) for a k-orbital atom, as a k x k table."""
    t = np.zeros((k, k), dtype=int)
    for a in range(k):
        for b in range(k):
            t[a, b] = dfo._pair1(a + 1, b + 1) - 1
    return t


def _reference_contraction(nat, first, last, n, nati, ptot_m, p_m, w):
    f = np.zeros((n, n))
    off, _ = dfo.partner_sizes(first, last, nati)
    ia = first[nati - 1] - 1
    ka = last[nati - 1] - first[nati - 1] + 1
    for jj, kk in off.items():
        ja = first[jj - 1] - 1
        kb = last[jj - 1] - first[jj - 1] + 1
        na_, nb_ = ka * (ka + 1) // 2, kb * (kb + 1) // 2
        blk = w[kk:kk + na_ * nb_].reshape(na_, nb_)
        T = blk[_pairs(ka)][:, :, _pairs(kb)]          # (mu, nu, lam, sig)
        PA = ptot_m[ia:ia + ka, ia:ia + ka]
        PB = ptot_m[ja:ja + kb, ja:ja + kb]
        pab = p_m[ia:ia + ka, ja:ja + kb]
        f[ia:ia + ka, ia:ia + ka] += np.einsum("mnls,ls->mn", T, PB)
        f[ja:ja + kb, ja:ja + kb] += np.einsum("mnls,mn->ls", T, PA)
        x = np.einsum("mnls,ns->ml", T, pab)
        f[ia:ia + ka, ja:ja + kb] -= x
        f[ja:ja + kb, ia:ia + ka] -= x.T
    r, c = np.tril_indices(n)
    return f[r, c]


@pytest.mark.parametrize("nat", [[8, 1, 1, 8, 1, 1], [6, 6, 1, 1, 1, 1, 1, 1, 1, 1], [1, 1, 1], [8, 6, 8]])
def test_dfock2_is_the_two_centre_contraction_of_the_atom(nat):
    rng = np.random.default_rng(len(nat))
    first, last, n = _layout(nat)
    ptot_m, ptot = _sym_packed(rng, n)
    p_m, p = _sym_packed(rng, n)
    for nati in range(1, len(nat) + 1):
        _, nw = dfo.partner_sizes(first, last, nati)
        w = rng.normal(size=nw)
        f = np.zeros(n * (n + 1) // 2)
        dfo.dfock2(f, ptot, p, w, first, last, nati)
        ref = _reference_contraction(nat, first, last, n, nati, ptot_m, p_m, w)
        assert np.abs(f - ref).max() < 1e-12 * max(1.0, np.abs(ref).max())
