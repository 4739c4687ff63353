"""The oracle's polychromatic structure factor (spsim's spectrum kernel,
src/diffraction.cu:415-476) against its own building blocks: no bandwidth or
one sample is the monochromatic sum, an even sample count above one is raised
by one, and with point scatterers (no form factor) the result is the
Gaussian-weighted mean of monochromatic patterns at the scaled q."""
import numpy as np

from conftest import golden
from oracle import oracle as O


def _case():
    g = golden("sf_small.npz")
    return g["Z"], g["pos"].astype(np.float64), g["hkl"].astype(np.float64)


def test_no_bandwidth_or_one_sample_is_monochromatic():
    Z, pos, q = _case()
    F, I = O.structure_factor(Z, pos, q)
    for bw, S in ((0.0, 5), (0.05, 1)):
        Fs, Is = O.structure_factor_spectrum(Z, pos, q, 2e-10, bw, S)
        assert np.array_equal(Fs, F) and np.array_equal(Is, I)


def test_even_sample_count_is_raised_by_one():
    Z, pos, q = _case()
    F4, _ = O.structure_factor_spectrum(Z, pos, q, 2e-10, 0.3, 4)
    F5, _ = O.structure_factor_spectrum(Z, pos, q, 2e-10, 0.3, 5)
    assert np.array_equal(F4, F5)


def test_weighted_mean_of_scaled_monochromatic_patterns():
    Z, pos, q = _case()
    lam, bw, S = 2e-10, 0.3, 7
    Fs, Is = O.structure_factor_spectrum(Z, pos, q, lam, bw, S, delta_atoms=True)
    sigma = (lam - lam * (1 - bw / 2)) / 2
    acc, tot = 0, 0
    for j in range(S):
        lj = lam * (1 - bw / 2) + j / (S - 1) * lam * bw
        w = np.exp(-((lj - lam) / sigma) ** 2 / 2)
        F, _ = O.structure_factor(Z, pos, q * (lam / lj), delta_atoms=True)
        acc = acc + w * F
        tot += w
    np.testing.assert_allclose(Fs, acc / tot, rtol=1e-12, atol=1e-12 * np.abs(Fs).max())
    np.testing.assert_allclose(Is, np.abs(Fs) ** 2, rtol=1e-12)
