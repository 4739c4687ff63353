"""Detector chain on the GPU against spsim's own outputs (golden fixtures) and
the oracle's copy of the Philox noise streams; noise statistics."""
import numpy as np
import pytest
import torch

from conftest import golden
from oracle import oracle as O
from spsim_b200 import core

pytestmark = pytest.mark.gpu


def _params(g, pol=0, spherical=0, readout=0.0, clamp=0, seed=0, pattern=0):
    p = g["params"]
    nx, ny, w, h, d, pw, ph, cx, cy, qe, eh, dark, fw, mv, bx, by, lam, I0, t = p
    return core.chain_params(nx=int(nx), ny=int(ny), width=w, height=h, distance=d, pixel_width=pw,
                             pixel_height=ph, center_x=cx, center_y=cy, quantum_efficiency=qe,
                             electron_hole_production_energy=eh, dark_current=dark, linear_full_well=fw,
                             maximum_value=mv, binning_x=int(bx), binning_y=int(by), wavelength=lam,
                             beam_intensity=I0, exposure_time=t, polarization=pol, spherical=spherical,
                             readout_noise=readout, clamp_to_maximum=clamp, seed=seed, pattern_index=pattern)


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


@pytest.mark.parametrize("pol", [0, 1, 2, 3])
def test_thomson_matches_reference(cuda, pol):
    g = golden("chain.npz")
    out = core.detector_chain(_params(g, pol=pol), None, outputs=["thomson_correction"])
    np.testing.assert_allclose(out["thomson_correction"].cpu().numpy(), g["thomson_%d" % pol], rtol=1.2e-7)


@pytest.mark.parametrize("sph", [0, 1])
def test_solid_angle_matches_reference(cuda, sph):
    g = golden("chain.npz")
    out = core.detector_chain(_params(g, spherical=sph), None, outputs=["solid_angle"])
    np.testing.assert_allclose(out["solid_angle"].cpu().numpy(), g["solid_angle_%d" % sph], rtol=2.4e-7)


def test_photons_electrons_and_binned_outputs_match_reference(cuda):
    from spsim_b200 import _native
    from spsim_b200.core import _dev, _stream_ptr

    g = golden("chain.npz")
    p = _params(g, pol=3)
    n = p.nx * p.ny
    L = _native.lib()
    T, Om, I = _t(g["thomson_3"]), _t(g["solid_angle_0"]), _t(g["ints"])
    ph = torch.empty(n, device="cuda")
    _native.check(L.spsim_b200_photons(n, _dev(T), _dev(Om), _dev(I), p.beam_intensity, _dev(ph), _stream_ptr()))
    np.testing.assert_allclose(ph.cpu().numpy(), g["photons"], rtol=1.2e-7)
    cnt = _t(g["counts"])
    el = torch.empty(n, device="cuda")
    _native.check(L.spsim_b200_electrons(p, _dev(cnt), _dev(el), _stream_ptr()))
    np.testing.assert_array_equal(el.cpu().numpy(), g["electrons"])
    nb = (p.nx // p.binning_x) * (p.ny // p.binning_y)
    ro, nl = torch.empty(nb, device="cuda"), torch.empty(nb, device="cuda")
    el_in, ph_in = _t(g["electrons"]), _t(g["photons"])  # keep the inputs alive across the launch
    _native.check(L.spsim_b200_binned_outputs(p, _dev(el_in), _dev(ph_in), _dev(ro), _dev(nl), _stream_ptr()))
    np.testing.assert_allclose(ro.cpu().numpy(), g["real_output"], rtol=1e-6)
    np.testing.assert_allclose(nl.cpu().numpy(), g["noiseless_output"], rtol=1e-6)


def test_fused_chain_agrees_with_stages(cuda):
    g = golden("chain.npz")
    p = _params(g, pol=3, readout=0.0, seed=11)
    out = core.detector_chain(p, _t(g["ints"]))
    ph = out["photons_per_pixel"].cpu().numpy()
    # T and Omega are recomputed in the fused kernel (each within an ulp of the reference's)
    np.testing.assert_allclose(ph, g["photons"], rtol=4e-7)
    counts = O.poisson(ph * np.float32(p.quantum_efficiency), seed=11)
    k = out["photon_count"].cpu().numpy()
    assert np.mean(k == counts) > 0.999
    hc = 1.98644521e-25
    epp = np.float32((hc / np.float64(np.float32(p.wavelength))) / np.float64(np.float32(
        p.electron_hole_production_energy)))
    np.testing.assert_array_equal(out["electrons_per_pixel"].cpu().numpy(), (k * epp).astype(np.float32))
    nl = O.noiseless_output(ph, p.nx, p.ny, p.binning_x, p.binning_y, np.float32(p.quantum_efficiency),
                            np.float32(p.wavelength), np.float32(p.electron_hole_production_energy),
                            p.linear_full_well, p.maximum_value)
    np.testing.assert_allclose(out["noiseless_output"].cpu().numpy(), nl, rtol=2e-6)


@pytest.mark.parametrize("lam", [0.05, 3.0, 9.99, 10.0, 37.0, 250.0, 999.0, 1000.0, 20000.0])
def test_poisson_stream_matches_oracle_and_moments(cuda, lam):
    n = 200000
    lam_a = np.full(n, lam, np.float32)
    k = core.poisson(_t(lam_a), seed=2024, pattern_index=3).cpu().numpy()
    ko = O.poisson(lam_a, seed=2024, pattern=3)
    assert np.mean(k == ko) > 0.999  # same Philox stream; fp32 math may differ in rare accept/reject ties
    se = np.sqrt(lam / n)
    assert abs(k.mean() - lam) < 6 * se + (0.5 if lam >= 1000 else 0)
    assert abs(k.var() / lam - 1) < 0.03
    assert np.all(k >= 0) and np.all(k == np.floor(k))


@pytest.mark.parametrize("lam", [2.5, 30.0, 300.0])
def test_poisson_chi_square(cuda, lam):
    from scipy import stats

    n = 400000
    k = core.poisson(_t(np.full(n, lam, np.float32)), seed=77).cpu().numpy().astype(int)
    lo, hi = int(stats.poisson.ppf(1e-4, lam)), int(stats.poisson.ppf(1 - 1e-4, lam))
    obs = np.array([(k < lo).sum()] + [(k == v).sum() for v in range(lo, hi + 1)] + [(k > hi).sum()])
    p = np.concatenate([[stats.poisson.cdf(lo - 1, lam)], stats.poisson.pmf(np.arange(lo, hi + 1), lam),
                        [stats.poisson.sf(hi, lam)]])
    exp = p * n
    keep = exp > 5
    chi2 = (((obs[keep] - exp[keep]) ** 2) / exp[keep]).sum()
    dof = keep.sum() - 1
    assert stats.chi2.sf(chi2, dof) > 1e-4, (chi2, dof)


def test_readout_noise_stream_and_clamp(cuda):
    nx = ny = 64
    p = core.chain_params(nx=nx, ny=ny, width=nx * 1e-4, height=ny * 1e-4, distance=0.1, pixel_width=1e-4,
                          pixel_height=1e-4, wavelength=1e-10, beam_intensity=0.0, quantum_efficiency=1.0,
                          electron_hole_production_energy=5.8e-19, dark_current=1e6, exposure_time=1.0,
                          readout_noise=10.0, linear_full_well=2e7, maximum_value=65535.0, clamp_to_maximum=1,
                          seed=99)
    out = core.detector_chain(p, torch.zeros(nx * ny, device="cuda"), outputs=["real_output"])
    ro = out["real_output"].cpu().numpy().astype(np.float64)
    noise = O.readout_noise(nx * ny, 10.0, seed=99)
    adc = np.float32(65535.0) / np.float32(2e7)
    expect = np.minimum(np.maximum(0, np.float32(1e6) + noise) * adc, 65535.0)
    assert np.mean(np.abs(ro - expect) <= 1e-6 * expect) > 0.999
    assert abs(np.std(ro / adc) - 10.0) < 0.5
    # clamp: a huge dark current saturates every pixel at maximum_value
    p.dark_current = 1e12
    out = core.detector_chain(p, torch.zeros(nx * ny, device="cuda"), outputs=["real_output"])
    assert float(out["real_output"].max()) == 65535.0


def test_binned_real_output_noise_is_per_binned_pixel(cuda):
    g = golden("chain.npz")
    p = _params(g, readout=5.0, seed=5)
    out = core.detector_chain(p, _t(g["ints"]))
    nb = (p.nx // p.binning_x) * (p.ny // p.binning_y)
    assert out["real_output"].numel() == nb
    base = O.real_output(out["electrons_per_pixel"].cpu().numpy(), O.readout_noise(nb, 5.0, seed=5), p.nx, p.ny,
                         p.binning_x, p.binning_y, np.float32(p.dark_current), np.float32(p.exposure_time),
                         p.linear_full_well, p.maximum_value)
    np.testing.assert_allclose(out["real_output"].cpu().numpy(), base, rtol=1e-5)
