"""The reference-shaped entry points (spsim.h, through the SWIG-mirror module)
against spsim's own outputs."""
import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden, intensity_errors
from oracle import oracle as O
from spsim_b200 import spsim as S

pytestmark = pytest.mark.gpu


def _mol(Z, pos):
    return S.get_molecule_from_atoms(Z, pos)


@pytest.mark.parametrize("fn", ["compute_pattern_on_list", "vector_compute_pattern_on_list",
                                "cuda_compute_pattern_on_list", "cuda_compute_pattern_on_list2"])
def test_compute_pattern_on_list_matches_reference(cuda, fn):
    g = golden("sf_small.npz")
    opts = S.set_defaults()
    opts.contents.verbosity_level = 0
    mol = _mol(g["Z"], g["pos"])
    n = g["hkl"].shape[0]
    pat = getattr(S, fn)(mol, g["hkl"], n, 0.0, opts.contents.experiment, opts)
    I = S.as_array(pat.contents.ints, n)
    F = S.as_array(pat.contents.F, n)
    e_max, e_l2 = intensity_errors(I, g["I"].astype(np.float64))
    assert e_max < 3e-5 and e_l2 < 3e-6
    assert np.abs(F - g["F"]).max() < 1e-5 * np.abs(g["F"]).max()
    np.testing.assert_array_equal(S.as_array(pat.contents.HKL_list, 3 * n), g["hkl"].reshape(-1))
    S.free_diffraction_pattern(pat)
    S.free_mol(mol)


def test_hkl_list_for_detector_bit_exact(cuda):
    g = golden("sf_small.npz")
    nx, ny, w, h, d, lam = g["det"]
    opts = S.set_defaults()
    det, exp = opts.contents.detector.contents, opts.contents.experiment.contents
    det.nx, det.ny, det.nz, det.width, det.height, det.distance = int(nx), int(ny), 1, w, h, d
    exp.wavelength = lam
    n = ctypes.c_int(0)
    for sph, key in ((0, "hkl"), (1, "hkl_spherical")):
        det.spherical = sph
        p = S.get_HKL_list_for_detector(opts.contents.detector, opts.contents.experiment, ctypes.byref(n))
        np.testing.assert_array_equal(S.as_array(p, 3 * n.value).reshape(-1, 3), g[key])
        ctypes.CDLL(None).free(ctypes.cast(p, ctypes.c_void_p))


def test_simulate_shot_chain_arrays(cuda, tmp_path):
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        opts = S.set_defaults()
        S.read_options_file(os.path.join(GOLDEN, "config", "example.conf"), opts)
        o = opts.contents
        det = o.detector.contents
        # keep it small: 64 x 64 pixels of the example's 40 um pitch
        det.width = det.height = 64 * det.pixel_width
        det.nx = det.ny = 64
        o.verbosity_level = 0
        g = golden("sf_small.npz")
        mol = _mol(g["Z"], g["pos"])
        pat = S.simulate_shot(mol, opts)
        n = 64 * 64
        I = S.as_array(pat.contents.ints, n)
        T = S.as_array(det.thomson_correction, n)
        Om = S.as_array(det.solid_angle, n)
        ph = S.as_array(det.photons_per_pixel, n)
        np.testing.assert_allclose(ph, (T * Om * I * np.float32(o.experiment.contents.beam_intensity)).astype(
            np.float32), rtol=1e-6)
        cnt = S.as_array(det.photon_count, n)
        assert np.all(cnt >= 0) and np.all(cnt == np.floor(cnt))
        nl = S.as_array(det.noiseless_output, n)
        assert np.all(np.isfinite(nl))
        ro = S.as_array(det.real_output, n)
        assert np.all(ro >= 0)
        assert pat.contents.rot
        S.free_stuff(pat, opts)
        S.free_mol(mol)
    finally:
        os.chdir(cwd)


def test_host_entry_point_reuses_scratch_safely(cuda):
    # repeated host-buffer calls: the same molecule with new HKL lists (the
    # molecule is reused), an edited copy of it (rebuilt), after a release
    from spsim_b200 import _native

    L = _native.lib()
    g = golden("sf_small.npz")
    Z = np.ascontiguousarray(g["Z"], np.int32)
    pos = np.ascontiguousarray(g["pos"], np.float32)
    hkl = np.ascontiguousarray(g["hkl"], np.float32)
    p = ctypes.c_void_p

    def call(Z, pos, hkl):
        n = hkl.shape[0]
        F = np.empty(2 * n, np.float32)
        I = np.empty(n, np.float32)
        st = L.spsim_b200_structure_factor_host(len(Z), Z.ctypes.data_as(p), pos.ctypes.data_as(p), None, None,
                                                ctypes.c_float(0), 0, None, ctypes.c_int64(n), hkl.ctypes.data_as(p),
                                                _native.PREC_F32, F.ctypes.data_as(p), I.ctypes.data_as(p))
        assert st == 0
        return I

    def want(Z, pos, hkl):
        return O.structure_factor(Z, pos.astype(np.float64), hkl.astype(np.float64))[1]

    cases = [(Z, pos, hkl), (Z, pos, hkl[::2].copy()), (Z, pos, (hkl * 0.7).astype(np.float32))]
    pos2 = pos.copy()
    pos2[3] += 1e-10  # one atom moved: the kept molecule must not be reused
    cases.append((Z, pos2, hkl))
    for Zc, pc, hc in cases:
        e_max, e_l2 = intensity_errors(call(Zc, pc, hc), want(Zc, pc, hc))
        assert e_max < 1e-5 and e_l2 < 1e-6, (e_max, e_l2)
    L.spsim_b200_release_scratch()
    e_max, _ = intensity_errors(call(Z, pos, hkl), want(Z, pos, hkl))
    assert e_max < 1e-5
