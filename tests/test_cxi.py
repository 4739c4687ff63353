"""CXI files of the spsim program's outputs (src/spsim.c:146-279), written by
the library's own HDF5 writer (no HDF5 library is in the image), read back
with an independent reader written from the HDF5 file format specification
(tests/h5read.py): layout, shapes, types, values and detector metadata.  CPU
only: output_array / output_carray run on the host."""
import ctypes
import os

import numpy as np
import pytest

import h5read
from spsim_b200 import spsim as S


def _opts(nx=24, ny=16, nz=1, binning=1):
    opts = S.set_defaults()
    d = opts.contents.detector.contents
    d.nx, d.ny, d.nz = nx, ny, nz
    d.binning_x = d.binning_y = binning
    d.binning_z = 1
    d.distance, d.pixel_width, d.pixel_height = 0.15, 75e-6, 80e-6
    opts.contents.experiment.contents.wavelength = 2.5e-10
    return opts


def test_real_array_file(tmp_path):
    os.chdir(tmp_path)
    opts = _opts()
    a = np.random.default_rng(1).normal(size=(16, 24)).astype(np.float32)
    S.output_array("photon_out", 3, a, None, opts)
    f = h5read.read(str(tmp_path / "photon_out-00003.cxi"))
    assert sorted(f) == ["/cxi_version", "/entry_1/image_1/data", "/entry_1/image_1/detector_1/distance",
                         "/entry_1/image_1/detector_1/x_pixel_size", "/entry_1/image_1/detector_1/y_pixel_size",
                         "/entry_1/image_1/mask", "/entry_1/image_1/source_1/wavelength"]
    assert f["/cxi_version"].dtype == np.int32 and int(f["/cxi_version"]) == 150
    data = f["/entry_1/image_1/data"]
    assert data.dtype == np.float32 and data.shape == (16, 24)
    np.testing.assert_array_equal(data, a)
    mask = f["/entry_1/image_1/mask"]
    assert mask.dtype == np.int32 and mask.shape == (16, 24) and np.all(mask == 1)
    assert float(f["/entry_1/image_1/detector_1/distance"]) == np.float32(0.15)
    assert float(f["/entry_1/image_1/detector_1/x_pixel_size"]) == np.float32(75e-6)
    assert float(f["/entry_1/image_1/detector_1/y_pixel_size"]) == np.float32(80e-6)
    assert float(f["/entry_1/image_1/source_1/wavelength"]) == np.float32(2.5e-10)


def test_complex_and_volume_files(tmp_path):
    os.chdir(tmp_path)
    opts = _opts(nx=8, ny=6, nz=5)
    rng = np.random.default_rng(2)
    c = (rng.normal(size=(5, 6, 8)) + 1j * rng.normal(size=(5, 6, 8))).astype(np.complex64)
    S.output_carray("scattering_factors", 0, c, None, opts)
    f = h5read.read(str(tmp_path / "scattering_factors-00000.cxi"))
    data = f["/entry_1/image_1/data"]
    assert data.shape == (5, 6, 8) and data.dtype.names == ("r", "i")
    np.testing.assert_array_equal(h5read.complex_of(data), c)


def test_orientation_and_binned_outputs(tmp_path):
    # a rotated shot carries its 3 x 3 orientation; binned detector outputs
    # keep their binned shape and pixel size
    os.chdir(tmp_path)
    opts = _opts(nx=24, ny=16, binning=2)
    R = np.array([[0, -1, 0], [1, 0, 0], [0, 0, 1]], np.float32)
    rot = S.SpRotation(3, 3, R.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    a = np.arange(24 * 16, dtype=np.float32).reshape(16, 24)
    S.output_array("solid_angles", 1, a, ctypes.pointer(rot), opts)
    f = h5read.read(str(tmp_path / "solid_angles-00001.cxi"))
    np.testing.assert_array_equal(f["/entry_1/image_1/orientation"], R.astype(np.float64))
    assert float(f["/entry_1/image_1/detector_1/x_pixel_size"]) == pytest.approx(2 * 75e-6, rel=1e-7)
    # the binned outputs through output_files: counts_out is (ny/2, nx/2)
    o = opts.contents
    for flag in ("output_scatt_int", "output_intensities", "output_sf_vtk", "output_noiseless_photons",
                 "output_scattering_factors", "output_solid_angles", "output_real_space", "output_photons",
                 "output_realspace_histogram"):
        setattr(o, flag, 0)
    o.output_count = o.output_noiseless_count = 1
    d = o.detector.contents
    counts = np.arange(12 * 8, dtype=np.float32)
    noiseless = counts * 0.5
    d.real_output = counts.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    d.noiseless_output = noiseless.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    ints = np.zeros(24 * 16, np.float32)
    pat = S.Diffraction_Pattern()
    pat.ints = ints.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    S.output_files(ctypes.pointer(pat), opts, 7)
    d.real_output = d.noiseless_output = None  # the arrays belong to this test
    for name, want in (("counts_out", counts), ("noiseless_counts_out", noiseless)):
        g = h5read.read(str(tmp_path / ("%s-00007.cxi" % name)))
        np.testing.assert_array_equal(g["/entry_1/image_1/data"], want.reshape(8, 12))
        assert float(g["/entry_1/image_1/detector_1/x_pixel_size"]) == pytest.approx(2 * 75e-6, rel=1e-7)
