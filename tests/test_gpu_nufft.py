"""NUFFT structure factor (spsim_b200_forward_nufft and the reference-shaped
compute_pattern_on_list_by_nfft / use_nfft_for_sf) against the FP64 direct
sum of the oracle.

Tolerances: relative L2 error of F below max(3 eps, 2e-7) (F is stored as
complex64, ~6e-8 relative rounding per component), maximum error below
max(30 eps, 2e-6) of max |F|; at the default eps = 1e-8 on the 50,000-atom
workload, the FP32 direct path's intensity tolerance (floored max 1e-5, L2
1e-6 against FP64)."""
import numpy as np
import pytest
import torch

from conftest import golden, intensity_errors
from oracle import oracle as O
from spsim_b200 import core, synth

pytestmark = pytest.mark.gpu


def _np(t):
    return t.cpu().numpy().astype(np.complex128 if t.is_complex() else np.float64)


def _check_F(F, F64, eps):
    rel = np.linalg.norm(F - F64) / np.linalg.norm(F64)
    mx = np.abs(F - F64).max() / np.abs(F64).max()
    assert rel < max(3 * eps, 2e-7), (eps, rel)
    assert mx < max(30 * eps, 2e-6), (eps, mx)
    return rel


@pytest.mark.parametrize("eps", [1e-3, 1e-6, 1e-9, 1e-12])
def test_small_molecule_meets_requested_eps(cuda, eps):
    g = golden("sf_small.npz")
    F64, I64 = O.structure_factor(g["Z"], g["pos"].astype(np.float64), g["hkl"].astype(np.float64))
    mol = core.Molecule(g["Z"], g["pos"])
    qs = core.QSet.from_list(g["hkl"])
    F, I = core.forward_nufft(mol, qs, eps=eps)
    core.synchronize()
    _check_F(_np(F), F64, eps)
    assert np.allclose(_np(I), np.abs(_np(F)) ** 2, rtol=1e-5, atol=1e-6 * I64.max())
    w1, w2, n2 = core.last_nufft_grid()
    assert w2 == min(max(int(np.ceil(-np.log10(eps))) + 1, 4), 15) and w1 == min(w2 + 3, 16)
    assert all(n % 2 == 0 and n >= 2 * (w2 + 3) for n in n2)


@pytest.mark.parametrize("kw", [{}, {"B": 30.0}, {"delta_atoms": True}, {"occ": True}, {"beam": True}],
                         ids=["plain", "B30", "delta", "occ", "beam"])
def test_rotated_detector_matches_oracle(cuda, kw):
    # 3,000 atoms on a 64 x 48 detector at two random orientations (the q box
    # and so the grid change with the rotation), global B, point atoms,
    # occupancies and a Gaussian beam (illumination weights)
    Z, pos = synth.random_molecule(3000, 4e-9, 7)
    rng = np.random.Generator(np.random.PCG64(8))
    occ = rng.uniform(-0.2, 1.0, len(Z)).astype(np.float32) if kw.get("occ") else None
    beam = (8e-9, 1e-9, -2e-9) if kw.get("beam") else None
    B = kw.get("B", 0.0)
    delta = kw.get("delta_atoms", False)
    d = dict(nx=64, ny=48, width=64 * 300e-6, height=48 * 300e-6, distance=0.08, wavelength=0.15e-9)
    q0 = O.hkl_detector(**d)
    mol = core.Molecule(Z, pos, occ=occ, delta_atoms=delta, beam=beam)
    qs = core.QSet.from_detector(**d)
    for r in synth.haar_rotations(2, 9):
        F, I = core.forward_nufft(mol, qs, rot=r, B=B, eps=1e-9)
        core.synchronize()
        F64, I64 = O.structure_factor(Z, pos.astype(np.float64), q0 @ r.T, occ=occ, B=B, delta_atoms=delta,
                                      beam=beam)
        _check_F(_np(F), F64, 1e-9)


def test_random_q_list_and_off_centre_molecule(cuda):
    # a q list with no detector structure (a full box of q) and a molecule
    # 50 nm from the origin: the centre phase is applied after the transform
    rng = np.random.Generator(np.random.PCG64(11))
    Z = rng.choice([1, 6, 7, 8, 16, 26], 700).astype(np.int32)
    pos = (rng.normal(size=(700, 3)) * 1e-9 + np.array([5e-8, -2e-8, 1e-8])).astype(np.float32)
    hkl = (rng.uniform(-1, 1, size=(5000, 3)) * 2e9).astype(np.float32)
    mol = core.Molecule(Z, pos)
    qs = core.QSet.from_list(hkl)
    F, I = core.forward_nufft(mol, qs, eps=1e-10)
    core.synchronize()
    F64, _ = O.structure_factor(Z, pos.astype(np.float64), hkl.astype(np.float64))
    _check_F(_np(F), F64, 1e-10)


def test_edge_cases(cuda):
    from spsim_b200._native import SpsimError, SPSIM_ERR_INVALID_ARG

    rng = np.random.Generator(np.random.PCG64(13))
    # one atom, one pixel; a flat q list (all q_z equal); skipped Z = 0 atoms
    for Z, hkl in [(np.array([6], np.int32), np.array([[1e9, 2e8, -3e7]], np.float32)),
                   (rng.choice([0, 6, 8], 50).astype(np.int32),
                    np.c_[rng.normal(size=(300, 2)) * 1e9, np.full(300, -1e8)].astype(np.float32))]:
        pos = (rng.normal(size=(len(Z), 3)) * 1e-9).astype(np.float32)
        F, I = core.forward_nufft(core.Molecule(Z, pos), core.QSet.from_list(hkl), eps=1e-9)
        core.synchronize()
        F64, _ = O.structure_factor(Z, pos.astype(np.float64), hkl.astype(np.float64))
        assert np.abs(_np(F) - F64).max() <= 2e-6 * max(1.0, np.abs(F64).max())
    # no atoms: zeros
    F, I = core.forward_nufft(core.Molecule(np.zeros(0, np.int32), np.zeros((0, 3), np.float32)),
                              core.QSet.from_list(np.ones((7, 3), np.float32) * 1e9))
    core.synchronize()
    assert not F.abs().any() and not I.any()
    # per-atom B factors and eps outside [1e-14, 1e-2] are rejected
    mol_b = core.Molecule(np.array([6, 8], np.int32), np.zeros((2, 3), np.float32), bfac=np.ones(2, np.float32))
    qs = core.QSet.from_list(np.ones((4, 3), np.float32) * 1e9)
    with pytest.raises(SpsimError) as e:
        core.forward_nufft(mol_b, qs)
    assert e.value.status == SPSIM_ERR_INVALID_ARG
    with pytest.raises(SpsimError):
        core.forward_nufft(core.Molecule(np.array([6], np.int32), np.zeros((1, 3), np.float32)), qs, eps=0.5)


def test_atoms_moved_outside_bounds_are_reported(cuda):
    from spsim_b200._native import SpsimError, SPSIM_ERR_RANGE

    Z, pos = synth.random_molecule(200, 1e-9, 15)
    mol = core.Molecule(Z, pos)
    qs = core.QSet.from_list((np.random.default_rng(3).normal(size=(500, 3)) * 1e9).astype(np.float32))
    moved = pos.astype(np.float64).copy()
    moved[0] += 2e-8  # far outside the creation-time radius and its margin
    mol.update_device(torch.from_numpy(moved).cuda())
    core.forward_nufft(mol, qs)
    with pytest.raises(SpsimError) as e:
        core.synchronize()
    assert e.value.status == SPSIM_ERR_RANGE
    core.synchronize()  # the error word is cleared once reported


def test_precision_50k_workload_meets_f32_tolerance(cuda):
    # the 50,000-atom / 1024^2 workload (every 64th detector row), default eps
    w = synth.WORKLOADS["precision_50k"]
    Z, pos = synth.random_molecule(w["natoms"], w["radius"], w["seed"])
    d = w["det"]
    q64 = O.hkl_detector(d["nx"], d["ny"], d["width"], d["height"], d["distance"], d["wavelength"])
    rows = np.arange(0, d["ny"], 64)
    sel = (rows[:, None] * d["nx"] + np.arange(d["nx"])[None, :]).reshape(-1)
    hkl = q64[sel].astype(np.float32)
    F64, I64 = O.structure_factor(Z, pos.astype(np.float64), hkl.astype(np.float64))
    F, I = core.forward_nufft(core.Molecule(Z, pos), core.QSet.from_list(hkl))
    core.synchronize()
    e_max, e_l2 = intensity_errors(_np(I), I64)
    print("nufft precision_50k rows vs FP64: floored max %.3g  L2 %.3g" % (e_max, e_l2))
    assert e_max < 1e-5 and e_l2 < 1e-6


def test_reference_shaped_nfft_path(cuda):
    # compute_pattern_on_list_by_nfft and compute_sf with use_nfft_for_sf:
    # unit atom weights, B, the HKL list copied into the result
    from spsim_b200 import spsim as S

    g = golden("sf_small.npz")
    opts = S.set_defaults()
    opts.contents.verbosity_level = 0
    mol = S.get_molecule_from_atoms(g["Z"], g["pos"])
    n = g["hkl"].shape[0]
    for B, ref in ((0.0, g["F"]), (20.0, g["F_B20"])):
        pat = S.compute_pattern_on_list_by_nfft(mol, g["hkl"], n, opts.contents.detector, B, opts)
        F = S.as_array(pat.contents.F, n)
        assert np.abs(F - ref).max() < 1e-5 * np.abs(ref).max()
        np.testing.assert_array_equal(S.as_array(pat.contents.HKL_list, 3 * n), g["hkl"].reshape(-1))
        S.free_diffraction_pattern(pat)
    opts.contents.use_nfft_for_sf = 1
    pat = S.compute_sf(mol, g["hkl"], n, opts)
    F = S.as_array(pat.contents.F, n)
    F64, _ = O.structure_factor(g["Z"], g["pos"].astype(np.float64), g["hkl"].astype(np.float64))
    assert np.linalg.norm(F - F64) / np.linalg.norm(F64) < 2e-7
    S.free_diffraction_pattern(pat)
    S.free_mol(mol)


def test_orientation_batch_matches_oracle_and_single_calls(cuda):
    # a batch of orientations on one grid sized for every rotation (the ball
    # |q| <= |q|max): each pattern as the oracle, and as single NUFFT calls
    Z, pos = synth.random_molecule(2500, 3.5e-9, 21)
    d = dict(nx=48, ny=40, width=48 * 300e-6, height=40 * 300e-6, distance=0.1, wavelength=0.2e-9)
    q0 = O.hkl_detector(**d)
    mol = core.Molecule(Z, pos)
    qs = core.QSet.from_detector(**d)
    R = synth.haar_rotations(5, 22)
    F, I = core.forward_nufft_batch(mol, qs, R, B=10.0)
    core.synchronize()
    assert F.shape == (5, qs.npix) and I.shape == (5, qs.npix)
    for i, r in enumerate(R):
        F64, _ = O.structure_factor(Z, pos.astype(np.float64), q0 @ r.T, B=10.0)
        _check_F(_np(F[i]), F64, 1e-8)
        Fs, _ = core.forward_nufft(mol, qs, rot=r, B=10.0)
        core.synchronize()
        assert np.abs(_np(Fs) - _np(F[i])).max() < 2e-6 * np.abs(F64).max()


def test_release_scratch_frees_and_rebuilds_the_grids(cuda):
    # spsim_b200_release_scratch drops the device's NUFFT grids and twiddle tables;
    # the next forward builds them again
    from spsim_b200._native import lib

    g = golden("sf_small.npz")
    mol = core.Molecule(g["Z"], g["pos"])
    qs = core.QSet.from_list(g["hkl"])
    F1, _ = core.forward_nufft(mol, qs)
    core.synchronize()
    F1 = _np(F1)
    lib().spsim_b200_release_scratch()
    F2, _ = core.forward_nufft(mol, qs)
    core.synchronize()
    assert np.abs(_np(F2) - F1).max() <= 1e-6 * np.abs(F1).max()


def _fft_size(n):
    m = max(n, 2)
    while True:
        if m % 2 == 0:
            r = m
            for f in (2, 3, 5, 7):
                while r % f == 0:
                    r //= f
            if r == 1:
                return m
        m += 1


def test_power_of_two_transforms_and_nine_elements(cuda):
    # the FFT passes take a padded shared-memory layout for power-of-two
    # lengths and interleave elements in groups of four (the last group of
    # nine elements holds one): a q box sized so that the transforms are 128
    # (x) and 256 (y) long, by the grid sizing of the library restated here
    # (n1 = ceil(2 r_bound 2 sigma1 S) + w1 + 2, even; n2 the next 2,3,5,7-smooth
    # even size of 2 n1)
    rng = np.random.Generator(np.random.PCG64(31))
    Z = rng.choice([1, 6, 7, 8, 15, 16, 26, 30, 34], 600).astype(np.int32)
    Z[:9] = [1, 6, 7, 8, 15, 16, 26, 30, 34]
    pos = (rng.normal(size=(600, 3)) * 1.2e-9).astype(np.float32)
    p = pos.astype(np.float64)
    c = 0.5 * (p.min(0) + p.max(0))
    rmax = np.sqrt(((p - c) ** 2).sum(1)).max()
    X = rmax + max(0.05 * rmax, 5e-10)
    S = np.array([49.5, 113.0, 30.0]) / (6.0 * X)
    q = rng.uniform(-1.0, 1.0, size=(4000, 3)) * S
    q[0], q[1] = -S, S  # the box's corners, so that its half-widths are S
    hkl = q.astype(np.float32)
    h = hkl.astype(np.float64)
    half = 0.5 * (h.max(0) - h.min(0))
    w2 = 9
    n1 = np.ceil(2.0 * X * 2.0 * 1.5 * half) + (w2 + 3) + 2
    n1 = n1 + n1 % 2
    want = tuple(_fft_size(int(np.ceil(2.0 * v))) for v in n1)
    assert want[0] == 128 and want[1] == 256
    F, I = core.forward_nufft(core.Molecule(Z, pos), core.QSet.from_list(hkl), eps=1e-8)
    core.synchronize()
    assert core.last_nufft_grid()[2] == want
    F64, _ = O.structure_factor(Z, pos.astype(np.float64), h)
    _check_F(_np(F), F64, 1e-8)


def test_tile_and_per_pixel_interpolation_give_the_same_bits(cuda):
    # the tile path (a 16 x 8 pixel tile's grid region in shared memory, every
    # pixel's x weights zero outside its stencil) against per-pixel stencil
    # reads: identical F on a detector, a rotated detector (single calls and a
    # batch) and a detector whose last tile row and column are partial
    Z, pos = synth.random_molecule(4000, 5e-9, 41)
    mol = core.Molecule(Z, pos)
    try:
        for nx, ny in ((96, 80), (77, 45)):
            qs = core.QSet.from_detector(nx, ny, nx * 300e-6, ny * 300e-6, 0.09, 0.16e-9)
            R = synth.haar_rotations(3, 43)
            runs = {}
            for mode in (1, 0):
                core.set_nufft_interp(mode)
                single = [core.forward_nufft(mol, qs, rot=r, eps=1e-8)[0] for r in (None, R[0])]
                batch = core.forward_nufft_batch(mol, qs, R, eps=1e-8)[0]
                core.synchronize()
                runs[mode] = [_np(f) for f in single] + [_np(batch)]
            for a, b in zip(runs[0], runs[1]):
                np.testing.assert_array_equal(a, b)
    finally:
        core.set_nufft_interp(0)
    with pytest.raises(Exception):
        core.set_nufft_interp(2)


def test_native_calls_on_another_thread_wait_for_a_pipelined_shot(cuda, tmp_path):
    # simulate_shot with use_nfft_for_sf in four row chunks reads the device's
    # NUFFT grids after the call that prepared them has returned; NUFFT
    # forwards of another molecule on another detector (other grid sizes),
    # issued meanwhile from this thread, wait until the shot's last chunk is
    # queued.  Each thread's results against its own single-threaded ones.
    import os
    import threading

    from conftest import GOLDEN
    from spsim_b200 import spsim as S

    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        opts = S.set_defaults()
        S.read_options_file(os.path.join(GOLDEN, "config", "example.conf"), opts)
        o = opts.contents
        det = o.detector.contents
        det.width, det.height = 256 * det.pixel_width, 256 * det.pixel_height
        det.nx, det.ny, det.nz = 256, 256, 1
        det.binning_x = det.binning_y = 1
        o.use_nfft_for_sf = 1
        o.verbosity_level = 0
        g = golden("sf_small.npz")
        smol = S.get_molecule_from_atoms(g["Z"], g["pos"])
        n = 256 * 256
        S.set_shot_chunks(4)

        def shot_I():
            shot = S.simulate_shot(smol, opts)
            I = S.as_array(shot.contents.ints, n).copy()
            S.free_stuff(shot, opts)
            return I

        I_ref = shot_I().astype(np.float64)
        Z2, pos2 = synth.random_molecule(6000, 6e-9, 53)
        mol2 = core.Molecule(Z2, pos2)
        qs2 = core.QSet.from_detector(160, 144, 160 * 200e-6, 144 * 200e-6, 0.12, 0.18e-9)
        F_ref, _ = core.forward_nufft(mol2, qs2, eps=1e-8)
        core.synchronize()
        F_ref = _np(F_ref)

        shots, errors = [], []

        def run_shots():
            try:
                for _ in range(4):
                    shots.append(shot_I())
            except Exception as e:  # reported below
                errors.append(e)

        t = threading.Thread(target=run_shots)
        t.start()
        forwards = []
        while t.is_alive() or len(forwards) < 4:
            F, _ = core.forward_nufft(mol2, qs2, eps=1e-8)
            core.synchronize()
            forwards.append(_np(F))
            if len(forwards) >= 60:
                break
        t.join()
        assert not errors, errors
        assert len(shots) == 4
        for I in shots:
            e_max, e_l2 = intensity_errors(I, I_ref)
            assert e_max < 1e-5 and e_l2 < 1e-6, (e_max, e_l2)
        for F in forwards:
            assert np.linalg.norm(F - F_ref) / np.linalg.norm(F_ref) < 1e-6
        S.free_mol(smol)
    finally:
        S.set_shot_chunks(0)
        os.chdir(cwd)
