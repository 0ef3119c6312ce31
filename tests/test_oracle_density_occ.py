"""The oracle's restatement of density_for_GPU (matrix/density_for_GPU.F90:
16-130) and densit (matrix/densit.F90) checked against itself: with occ = 2
and orthonormal MOs the positron equivalent (the virtual and open MOs
subtracted from occ * I) and the electron equivalent are the same matrix, in
both the DGEMM form (iopc 3) and the explicit sums (iopc 6)."""
import numpy as np
import pytest

from oracle import scf_oracle as so


def _mos(n, seed=3):
    return np.linalg.qr(np.random.default_rng(seed).normal(size=(n, n)))[0]


@pytest.mark.parametrize("iopc", [3, 6])
@pytest.mark.parametrize("ndubl,nsingl,fract", [(14, 27, 0.5), (20, 31, 1.0), (9, 40, 1.5)])
def test_positron_and_electron_equivalents_agree(iopc, ndubl, nsingl, fract):
    n = 48
    c = _mos(n)
    pos = so.density_for_gpu(c, fract, ndubl, nsingl, 2.0, 1, iopc)   # mode 1: positron allowed
    ele = so.density_for_gpu(c, fract, ndubl, nsingl, 2.0, 2, iopc)   # mode 2: electron only
    ref = so.pack(2.0 * c[:, :ndubl] @ c[:, :ndubl].T + fract * c[:, ndubl:nsingl] @ c[:, ndubl:nsingl].T)
    np.testing.assert_allclose(ele, ref, atol=1e-12)
    if nsingl > n // 2:
        np.testing.assert_allclose(pos, ref, atol=1e-12)


def test_closed_shell_forms_agree_and_small_fractions_follow_the_iopc():
    n, k = 40, 13
    c = _mos(n, 5)
    closed = so.density(c, k)
    for iopc in (2, 3, 4, 5, 6):
        np.testing.assert_allclose(so.density_for_gpu(c, 0.0, k, k, 2.0, 1, iopc), closed, atol=1e-13)
    # a fraction below 0.01: iopc 5 keeps dsyrk's closed-shell product, the
    # explicit sums (densit) keep the fractional MOs
    small = 0.005
    p5 = so.density_for_gpu(c, small, k, k + 2, 2.0, 1, 5)
    p6 = so.density_for_gpu(c, small, k, k + 2, 2.0, 1, 6)
    np.testing.assert_allclose(p5, closed, atol=1e-13)
    np.testing.assert_allclose(p6 - closed, so.pack(small * c[:, k:k + 2] @ c[:, k:k + 2].T), atol=1e-13)


def test_uhf_spin_density_in_the_dgemm_form_doubles_the_full_orbitals():
    """density_for_GPU's DGEMM form weighs the fully occupied MOs by 2*sign
    whatever occ is (:63, :79); a UHF spin (occ = 1) with open MOs therefore
    gets 2 C_d C_d^T + fract C_o C_o^T there, and occ * C_d C_d^T in dsyrk's
    form (iopc 5 below fract 0.01)."""
    n = 30
    c = _mos(n, 7)
    p3 = so.density_for_gpu(c, 0.5, 8, 10, 1.0, 1, 3)
    np.testing.assert_allclose(p3, so.pack(2.0 * c[:, :8] @ c[:, :8].T + 0.5 * c[:, 8:10] @ c[:, 8:10].T),
                               atol=1e-13)
    p5 = so.density_for_gpu(c, 0.0, 8, 8, 1.0, 1, 5)
    np.testing.assert_allclose(p5, so.pack(c[:, :8] @ c[:, :8].T), atol=1e-13)
