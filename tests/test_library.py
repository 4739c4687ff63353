"""The C-ABI library: built in-tree, loads without a GPU, exports exactly the
functions include/*.h declares, and refuses work cleanly when no device is
present.  No compute calls (CPU only)."""
import ctypes
import subprocess

import pytest

from spsim_b200 import _native
from spsim_b200.build import exported_symbols, lib_path


def test_library_is_built_in_tree():
    import os

    assert os.path.exists(lib_path()), "run python -m spsim_b200.build"
    assert "spsim_b200/_lib" in lib_path()


def test_exports_every_declared_symbol_and_nothing_else():
    declared = set(exported_symbols())
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path()], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if line.split()[-2] in ("T", "W")}
    assert declared, "no declarations parsed from include/*.h"
    assert declared == exported, (sorted(declared - exported), sorted(exported - declared))


def test_reference_entry_points_are_declared():
    # the names spsim's SWIG module and C callers bind (include/diffraction.h, spsim.h, config.h, ...)
    need = {"compute_pattern_on_list", "vector_compute_pattern_on_list", "cuda_compute_pattern_on_list",
            "cuda_compute_pattern_on_list2", "get_HKL_list_for_detector", "apply_orientation_to_HKL_list",
            "calculate_thomson_correction", "calculate_pixel_solid_angle", "calculate_photons_per_pixel",
            "generate_poisson_noise", "calculate_electrons_per_pixel", "calculate_real_detector_output",
            "calculate_noiseless_detector_output", "compute_sf", "simulate_shot", "set_defaults",
            "read_options_file", "write_options_file", "free_diffraction_pattern", "free_output_in_options",
            "alloc_mol", "add_atom_to_mol", "get_HKL_list"}
    assert need <= set(exported_symbols())


def test_library_loads_and_reports_version():
    assert "sm_100a" in _native.version()


def test_status_strings():
    L = _native.lib()
    assert L.spsim_b200_status_string(0) == b"ok"
    assert b"phase range" in L.spsim_b200_status_string(_native.SPSIM_ERR_RANGE)


def _has_gpu():
    return _native.device_count() > 0


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_no_device_is_an_error_not_a_fallback():
    n = _native.device_count()
    assert n == 0
    with pytest.raises(_native.SpsimError) as e:
        _native.check(_native.lib().spsim_b200_init(0))
    assert e.value.status == _native.SPSIM_ERR_NO_DEVICE
    h = ctypes.c_void_p()
    import numpy as np

    Z = np.array([6], np.int32)
    pos = np.zeros(3, np.float32)
    st = _native.lib().spsim_b200_molecule_create(1, Z.ctypes.data_as(ctypes.c_void_p),
                                                  pos.ctypes.data_as(ctypes.c_void_p), None, None, 0, None,
                                                  ctypes.byref(h))
    assert st == _native.SPSIM_ERR_NO_DEVICE


def test_invalid_arguments_rejected_before_device_use():
    L = _native.lib()
    h = ctypes.c_void_p()
    assert L.spsim_b200_molecule_create(-1, None, None, None, None, 0, None, ctypes.byref(h)) == \
        _native.SPSIM_ERR_INVALID_ARG
    assert L.spsim_b200_qset_from_detector(0, 5, 1.0, 1.0, 1.0, 0.0, 0.0, 1e-10, 0, ctypes.byref(h)) == \
        _native.SPSIM_ERR_INVALID_ARG
    p = _native.ChainParams(nx=4, ny=4, nz=1, binning_x=0, binning_y=1, binning_z=1)
    assert L.spsim_b200_thomson(ctypes.byref(p), None, None) == _native.SPSIM_ERR_INVALID_ARG
    # the NUFFT forwards: NULL handles, and a batch outside [1, 65535] patterns
    assert L.spsim_b200_forward_nufft(None, None, None, 0.0, 1e-8, None, None, None) == _native.SPSIM_ERR_INVALID_ARG
    assert L.spsim_b200_forward_nufft_batch(None, None, 0, None, 0.0, 1e-8, None, None, None) == \
        _native.SPSIM_ERR_INVALID_ARG


def test_legacy_nufft_eps_setting():
    # the relative error used by compute_pattern_on_list_by_nfft / use_nfft_for_sf
    from spsim_b200 import spsim as S

    assert S.get_nufft_eps() == 1e-8
    try:
        S.set_nufft_eps(1e-10)
        assert S.get_nufft_eps() == 1e-10
    finally:
        S.set_nufft_eps(1e-8)


def test_shot_chunk_setting_is_clamped():
    # simulate_shot's row chunks: 0 automatic, 1 none, at most 8; negative
    # values mean automatic (no device needed)
    from spsim_b200 import spsim as S

    assert S.get_shot_chunks() == 0
    try:
        for v, want in ((3, 3), (1, 1), (20, 8), (-5, 0)):
            S.set_shot_chunks(v)
            assert S.get_shot_chunks() == want
    finally:
        S.set_shot_chunks(0)
