"""3-D (volume) detectors: the GPU grid bit for bit against spsim's own
get_HKL_list_for_3d_detector, and simulate_shot on a volume against the FP64
oracle (structure factor) with the chain arrays sized nx*ny*nz."""
import ctypes

import numpy as np
import pytest

from conftest import intensity_errors
from oracle import oracle as O
from spsim_b200 import spsim as S
from spsim_b200 import synth

pytestmark = pytest.mark.gpu


def _opts(nx, ny, nz):
    opts = S.set_defaults()
    o = opts.contents
    o.verbosity_level = 0
    det, exp = o.detector.contents, o.experiment.contents
    det.nx, det.ny, det.nz = nx, ny, nz
    det.width, det.height, det.depth = 1.2e-2, 9e-3, 6e-3
    det.pixel_width, det.pixel_height, det.pixel_depth = 1.2e-2 / nx, 9e-3 / ny, 6e-3 / nz
    det.distance = 0.1
    det.center_x, det.center_y, det.center_z = 1e-4, -5e-5, 2e-5
    det.binning_x = det.binning_y = det.binning_z = 1
    det.quantum_efficiency, det.electron_hole_production_energy = 1.0, 5.8e-19
    det.linear_full_well, det.maximum_value = 2e5, 65535.0
    exp.wavelength, exp.beam_intensity, exp.exposure_time = 2e-10, 1e30, 1e-3
    o.random_seed = 3
    return opts


def test_volume_grid_bit_exact_against_reference(cuda):
    nx, ny, nz = 24, 20, 12
    opts = _opts(nx, ny, nz)
    n = ctypes.c_int(0)
    p = S.get_HKL_list_for_3d_detector(opts.contents.detector, opts.contents.experiment, ctypes.byref(n))
    ours = S.as_array(p, 3 * n.value).reshape(-1, 3)
    ctypes.CDLL(None).free(ctypes.cast(p, ctypes.c_void_p))
    want = O.hkl_3d_detector(nx, ny, nz, 1.2e-2, 9e-3, 6e-3, 0.1, 2e-10, center=(1e-4, -5e-5, 2e-5))
    assert n.value == nx * ny * nz
    assert np.array_equal(ours.view(np.uint32), want.view(np.uint32))


def test_simulate_shot_on_a_volume(cuda):
    nx, ny, nz = 16, 12, 8
    opts = _opts(nx, ny, nz)
    Z, pos = synth.random_molecule(800, 2e-9, 9)
    mol = S.get_molecule_from_atoms(Z, pos)
    pat = S.simulate_shot(mol, opts)
    n = nx * ny * nz
    I = S.as_array(pat.contents.ints, n)
    q = O.hkl_3d_detector(nx, ny, nz, 1.2e-2, 9e-3, 6e-3, 0.1, 2e-10, center=(1e-4, -5e-5, 2e-5))
    _, I64 = O.structure_factor(Z, pos.astype(np.float64), q.astype(np.float64))
    e_max, e_l2 = intensity_errors(I, I64)
    assert e_max < 1e-5 and e_l2 < 1e-6, (e_max, e_l2)
    det = opts.contents.detector.contents
    om = S.as_array(det.solid_angle, n)
    np.testing.assert_allclose(om, np.float32(det.pixel_width * det.pixel_height / 0.1 ** 2), rtol=1e-6)
    for arr in (det.photons_per_pixel, det.photon_count, det.real_output, det.noiseless_output):
        assert np.all(np.isfinite(S.as_array(arr, n)))
    S.free_stuff(pat, opts)
    S.free_mol(mol)
