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


@pytest.mark.parametrize("use_cuda,bandwidth,nfft", [(1, 0.0, 0), (2, 0.0, 0), (1, 0.3, 0), (2, 0.3, 0), (1, 0.0, 1)],
                         ids=["cuda1", "cuda2", "cuda1_bw", "cuda2_bw", "nfft"])
def test_simulate_shot_equals_step_by_step_sequence(cuda, tmp_path, use_cuda, bandwidth, nfft):
    # simulate_shot runs geometry, orientation, structure factor and the chain
    # as one device pipeline; its outputs must be those of the reference's
    # step-by-step sequence (src/spsim.c:281-346) through the public calls:
    # HKL list bit for bit (device rotation = host float loop), F and |F|^2
    # bit for bit (to 1e-6 of the maximum for the NUFFT, whose spreading adds
    # in FP64 atomics of unspecified order), the chain arrays as the fused
    # chain gives them (within a few ulps of the per-stage functions; noise
    # from the same streams)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        opts = S.set_defaults()
        S.read_options_file(os.path.join(GOLDEN, "config", "example.conf"), opts)
        o = opts.contents
        det, exp = o.detector.contents, o.experiment.contents
        det.width = det.height = 48 * det.pixel_width
        det.nx = det.ny = 48
        det.readout_noise = 3.0
        o.verbosity_level = 0
        o.use_cuda = use_cuda  # 1: the spectrum path when there is a bandwidth
        o.use_nfft_for_sf = nfft
        o.wavelength_samples = 4
        exp.bandwidth = bandwidth
        o.random_orientation = 0
        o.euler_orientation[0], o.euler_orientation[1], o.euler_orientation[2] = 0.3, -1.1, 2.2
        o.random_seed = 4242
        S.set_noise_seed(4242)
        g = golden("sf_small.npz")
        mol = _mol(g["Z"], g["pos"])
        n = 48 * 48

        # the reference sequence, step by step (no pattern counter step in between)
        size = ctypes.c_int(0)
        hkl = S.get_HKL_list(opts, ctypes.byref(size))
        hp = ctypes.pointer(hkl)
        rot = S.apply_orientation_to_HKL_list(hp, ctypes.byref(size), opts)
        pat = S.compute_sf(mol, hp.contents, size.value, opts)
        S.calculate_thomson_correction(o.detector, o.experiment)
        S.calculate_pixel_solid_angle(o.detector)
        S.calculate_photons_per_pixel(pat, opts)
        S.generate_poisson_noise(o.detector)
        S.calculate_electrons_per_pixel(o.detector, o.experiment)
        S.calculate_real_detector_output(o.detector, o.experiment)
        S.calculate_noiseless_detector_output(o.detector, o.experiment)
        names = ["thomson_correction", "solid_angle", "photons_per_pixel", "photon_count", "electrons_per_pixel",
                 "real_output", "noiseless_output"]
        step = {k: S.as_array(getattr(det, k), n).copy() for k in names}
        step_hkl = S.as_array(pat.contents.HKL_list, 3 * n).copy()
        step_F = S.as_array(pat.contents.F, n).copy()
        step_I = S.as_array(pat.contents.ints, n).copy()
        step_rot = np.ctypeslib.as_array(rot.contents.data, shape=(9,)).copy()
        S.free_diffraction_pattern(pat)
        S.free_output_in_options(opts)

        shot = S.simulate_shot(mol, opts)
        np.testing.assert_array_equal(S.as_array(shot.contents.HKL_list, 3 * n), step_hkl)
        np.testing.assert_array_equal(np.ctypeslib.as_array(shot.contents.rot.contents.data, shape=(9,)), step_rot)
        if nfft:
            assert np.abs(S.as_array(shot.contents.F, n) - step_F).max() <= 1e-6 * np.abs(step_F).max()
            assert np.abs(S.as_array(shot.contents.ints, n) - step_I).max() <= 2e-6 * step_I.max()
            F64, _ = O.structure_factor(g["Z"], g["pos"].astype(np.float64), step_hkl.reshape(-1, 3).astype(np.float64))
            assert np.linalg.norm(step_F - F64) / np.linalg.norm(F64) < 2e-7
        else:
            np.testing.assert_array_equal(S.as_array(shot.contents.F, n), step_F)
            np.testing.assert_array_equal(S.as_array(shot.contents.ints, n), step_I)
        got = {k: S.as_array(getattr(det, k), n) for k in names}
        np.testing.assert_allclose(got["thomson_correction"], step["thomson_correction"], rtol=2.4e-7)
        np.testing.assert_allclose(got["solid_angle"], step["solid_angle"], rtol=2.4e-7)
        np.testing.assert_allclose(got["photons_per_pixel"], step["photons_per_pixel"], rtol=6e-7)
        np.testing.assert_allclose(got["noiseless_output"], step["noiseless_output"], rtol=1e-6)
        assert np.mean(got["photon_count"] == step["photon_count"]) > 0.995
        same = got["photon_count"] == step["photon_count"]
        np.testing.assert_allclose(got["electrons_per_pixel"][same], step["electrons_per_pixel"][same], rtol=1e-6)
        np.testing.assert_allclose(got["real_output"][same], step["real_output"][same], rtol=1e-5, atol=1e-3)
        assert shot.contents.HKL_list_size == n
        S.free_stuff(shot, opts)
        S.free_mol(mol)
    finally:
        os.chdir(cwd)


def _shot_arrays(shot, det, n, nb):
    names = ["thomson_correction", "solid_angle", "photons_per_pixel", "photon_count", "electrons_per_pixel"]
    out = {k: S.as_array(getattr(det, k), n).copy() for k in names}
    for k in ("real_output", "noiseless_output"):
        out[k] = S.as_array(getattr(det, k), nb).copy()
    out["F"] = S.as_array(shot.contents.F, n).copy()
    out["I"] = S.as_array(shot.contents.ints, n).copy()
    out["hkl"] = S.as_array(shot.contents.HKL_list, 3 * n).copy()
    return out


@pytest.mark.parametrize("nx,ny,binning,spherical,polarization,nfft",
                         [(96, 90, 1, 0, 0, 0), (95, 91, 2, 0, 0, 0), (64, 64, 2, 0, 0, 0), (80, 72, 1, 1, 3, 0),
                          (72, 81, 3, 0, 1, 0), (96, 90, 1, 0, 0, 1), (77, 70, 2, 0, 0, 1)],
                         ids=["even", "odd_binned", "square_binned", "spherical_unpolarised", "vertical_binned3",
                              "nufft", "nufft_odd_binned"])
def test_simulate_shot_row_chunks_match_step_by_step(cuda, tmp_path, nx, ny, binning, spherical, polarization, nfft):
    # the pipelined simulate_shot (three row chunks on two streams, each
    # chunk's outputs copied while the next computes) against the reference's
    # step-by-step sequence on the whole detector (no pattern counter step in
    # between, so both draw the same noise streams): the HKL list and the
    # geometry-only chain arrays bit for bit, |F|^2 within the FP32 tolerance
    # of the one-pass result and of the FP64 oracle (the chunks split their
    # atom ranges differently), the noise stages where the counts agree
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        opts = S.set_defaults()
        S.read_options_file(os.path.join(GOLDEN, "config", "example.conf"), opts)
        o = opts.contents
        det = o.detector.contents
        det.width, det.height = nx * det.pixel_width, ny * det.pixel_height
        det.nx, det.ny, det.nz = nx, ny, 1
        det.binning_x = det.binning_y = binning
        det.spherical = spherical
        o.experiment.contents.polarization = polarization
        o.use_nfft_for_sf = nfft  # the NUFFT: one grid, the chunks' interpolations in turn
        det.readout_noise = 3.0
        o.verbosity_level = 0
        o.random_orientation = 0
        o.euler_orientation[0], o.euler_orientation[1], o.euler_orientation[2] = 0.3, -1.1, 2.2
        o.random_seed = 77
        S.set_noise_seed(77)
        g = golden("sf_small.npz")
        mol = _mol(g["Z"], g["pos"])
        n, nb = nx * ny, (nx // binning) * (ny // binning)

        size = ctypes.c_int(0)
        hkl = S.get_HKL_list(opts, ctypes.byref(size))
        hp = ctypes.pointer(hkl)
        rot = S.apply_orientation_to_HKL_list(hp, ctypes.byref(size), opts)
        pat = S.compute_sf(mol, hp.contents, size.value, opts)
        S.calculate_thomson_correction(o.detector, o.experiment)
        S.calculate_pixel_solid_angle(o.detector)
        S.calculate_photons_per_pixel(pat, opts)
        S.generate_poisson_noise(o.detector)
        S.calculate_electrons_per_pixel(o.detector, o.experiment)
        S.calculate_real_detector_output(o.detector, o.experiment)
        S.calculate_noiseless_detector_output(o.detector, o.experiment)
        one = _shot_arrays(pat, det, n, nb)
        S.free_diffraction_pattern(pat)
        S.free_output_in_options(opts)

        S.set_shot_chunks(3)
        shot = S.simulate_shot(mol, opts)
        S.set_shot_chunks(0)
        ch = _shot_arrays(shot, det, n, nb)
        S.free_stuff(shot, opts)

        np.testing.assert_array_equal(ch["hkl"], one["hkl"])
        np.testing.assert_allclose(ch["thomson_correction"], one["thomson_correction"], rtol=2.4e-7)
        np.testing.assert_allclose(ch["solid_angle"], one["solid_angle"], rtol=2.4e-7)
        e_max, e_l2 = intensity_errors(ch["I"], one["I"].astype(np.float64))
        assert e_max < 1e-5 and e_l2 < 1e-6, (e_max, e_l2)
        _, I64 = O.structure_factor(g["Z"], g["pos"].astype(np.float64), ch["hkl"].reshape(-1, 3).astype(np.float64))
        e_max, e_l2 = intensity_errors(ch["I"], I64)
        assert e_max < 1e-5 and e_l2 < 1e-6, (e_max, e_l2)
        np.testing.assert_allclose(ch["photons_per_pixel"], one["photons_per_pixel"], rtol=2e-5)
        same = ch["photon_count"] == one["photon_count"]
        assert same.mean() > 0.995
        np.testing.assert_allclose(ch["electrons_per_pixel"][same], one["electrons_per_pixel"][same], rtol=1e-6)
        np.testing.assert_allclose(ch["noiseless_output"], one["noiseless_output"], rtol=2e-5, atol=1e-6)
        if binning == 1:
            np.testing.assert_allclose(ch["real_output"][same], one["real_output"][same], rtol=1e-5, atol=1e-3)
        else:
            # a bin's real output sums its pixels' electrons: compared where every pixel's count agrees
            cnt = same.reshape(ny, nx)[: ny // binning * binning, : nx // binning * binning]
            bins_same = cnt.reshape(ny // binning, binning, nx // binning, binning).all(axis=(1, 3)).reshape(-1)
            assert bins_same.mean() > 0.98
            np.testing.assert_allclose(ch["real_output"][bins_same], one["real_output"][bins_same], rtol=1e-5,
                                       atol=1e-3)
        S.free_mol(mol)
    finally:
        S.set_shot_chunks(0)
        os.chdir(cwd)


@pytest.mark.parametrize("nfft", [0, 1])
def test_simulate_shot_row_chunks_without_atoms(cuda, tmp_path, nfft):
    # a molecule whose atoms are all Z = 0 (skipped, src/diffraction.c:830-832)
    # through the pipelined shot, direct and NUFFT: every chunk's F and |F|^2
    # are zeros, and the HKL list and geometry arrays those of one pass
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        opts = S.set_defaults()
        S.read_options_file(os.path.join(GOLDEN, "config", "example.conf"), opts)
        o = opts.contents
        det = o.detector.contents
        nx, ny = 64, 60
        det.width, det.height = nx * det.pixel_width, ny * det.pixel_height
        det.nx, det.ny, det.nz = nx, ny, 1
        det.binning_x = det.binning_y = 1
        o.use_nfft_for_sf = nfft
        o.verbosity_level = 0
        o.random_seed = 5
        mol = _mol(np.zeros(5, np.int32), np.linspace(-1e-9, 1e-9, 15).reshape(5, 3))
        n, nb = nx * ny, nx * ny
        out = {}
        for chunks in (1, 3):
            S.set_shot_chunks(chunks)
            shot = S.simulate_shot(mol, opts)
            out[chunks] = _shot_arrays(shot, det, n, nb)
            S.free_stuff(shot, opts)
        ch, one = out[3], out[1]
        assert not ch["F"].any() and not ch["I"].any()
        assert not ch["photons_per_pixel"].any() and not ch["photon_count"].any()
        np.testing.assert_array_equal(ch["hkl"], one["hkl"])
        np.testing.assert_array_equal(ch["solid_angle"], one["solid_angle"])
        S.free_mol(mol)
    finally:
        S.set_shot_chunks(0)
        os.chdir(cwd)


def test_simulate_shot_automatic_chunks_on_a_large_detector(cuda, tmp_path):
    # 1024 x 512 pixels (2^19): simulate_shot pipelines four row chunks by
    # default; every 29th row against the FP64 oracle, the chain's geometry
    # arrays against the per-stage calls
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        assert S.get_shot_chunks() == 0
        opts = S.set_defaults()
        S.read_options_file(os.path.join(GOLDEN, "config", "example.conf"), opts)
        o = opts.contents
        det = o.detector.contents
        nx, ny = 1024, 512
        det.width, det.height = nx * det.pixel_width, ny * det.pixel_height
        det.nx, det.ny, det.nz = nx, ny, 1
        o.verbosity_level = 0
        g = golden("sf_small.npz")
        mol = _mol(g["Z"], g["pos"])
        shot = S.simulate_shot(mol, opts)
        n = nx * ny
        I = S.as_array(shot.contents.ints, n).reshape(ny, nx)
        hkl = S.as_array(shot.contents.HKL_list, 3 * n).reshape(ny, nx, 3)
        rows = np.arange(0, ny, 29)
        _, I64 = O.structure_factor(g["Z"], g["pos"].astype(np.float64), hkl[rows].reshape(-1, 3).astype(np.float64))
        e_max, e_l2 = intensity_errors(I[rows].reshape(-1), I64)
        assert e_max < 1e-5 and e_l2 < 1e-6, (e_max, e_l2)
        T = S.as_array(det.thomson_correction, n).copy()
        Om = S.as_array(det.solid_angle, n).copy()
        ph = S.as_array(det.photons_per_pixel, n)
        np.testing.assert_allclose(ph, (T * Om * I.reshape(-1) * np.float32(o.experiment.contents.beam_intensity)),
                                   rtol=1e-6)
        S.free_stuff(shot, opts)
        S.calculate_thomson_correction(o.detector, o.experiment)
        S.calculate_pixel_solid_angle(o.detector)
        np.testing.assert_array_equal(S.as_array(det.thomson_correction, n), T)
        np.testing.assert_array_equal(S.as_array(det.solid_angle, n), Om)
        S.free_output_in_options(opts)
        S.free_mol(mol)
    finally:
        os.chdir(cwd)
