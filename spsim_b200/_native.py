"""ctypes binding of libspsim_b200.so (include/spsim_b200.h and include/spsim.h).

The library is the in-tree build under spsim_b200/_lib/.  Loading fails loudly
when it is missing: there is no Python or CPU fallback for any kernel.
"""
import ctypes
import os
import threading

from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_int64, c_uint32, c_uint64, c_void_p

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libspsim_b200.so")

SPSIM_OK = 0
SPSIM_ERR_INVALID_ARG = 1
SPSIM_ERR_CUDA = 2
SPSIM_ERR_NO_DEVICE = 3
SPSIM_ERR_OUT_OF_MEMORY = 4
SPSIM_ERR_RANGE = 5
SPSIM_ERR_TIMEOUT = 6
SPSIM_ERR_UNSUPPORTED = 7

PREC_FP64 = 0
PREC_F32 = 1
PREC_F32_FAST = 2
PRECISIONS = {"fp64": PREC_FP64, "f32": PREC_F32, "f32_fast": PREC_F32_FAST}

MEM_HOST = 0
MEM_DEVICE = 1


class SpsimError(RuntimeError):
    """A non-zero status from the native library."""

    def __init__(self, status, message):
        super().__init__("%s (status %d): %s" % (_status_name(status), status, message))
        self.status = status


def _status_name(status):
    try:
        return lib().spsim_b200_status_string(status).decode()
    except Exception:  # noqa: BLE001 - only used while formatting an error
        return "error"


class ChainParams(ctypes.Structure):
    """spsim_b200_chain_params."""

    _fields_ = [
        ("nx", c_int), ("ny", c_int), ("nz", c_int),
        ("binning_x", c_int), ("binning_y", c_int), ("binning_z", c_int),
        ("spherical", c_int), ("polarization", c_int),
        ("width", c_float), ("height", c_float), ("distance", c_float),
        ("center_x", c_float), ("center_y", c_float),
        ("pixel_width", c_float), ("pixel_height", c_float),
        ("wavelength", c_float), ("beam_intensity", c_float),
        ("quantum_efficiency", c_float), ("electron_hole_production_energy", c_float),
        ("dark_current", c_float), ("exposure_time", c_float), ("readout_noise", c_float),
        ("linear_full_well", c_float), ("maximum_value", c_float),
        ("clamp_to_maximum", c_int),
        ("seed", c_uint64), ("pattern_index", c_uint32),
    ]


class ChainOutputs(ctypes.Structure):
    """spsim_b200_chain_outputs (device pointers)."""

    _fields_ = [
        ("thomson_correction", c_void_p), ("solid_angle", c_void_p), ("photons_per_pixel", c_void_p),
        ("photon_count", c_void_p), ("electrons_per_pixel", c_void_p), ("real_output", c_void_p),
        ("noiseless_output", c_void_p),
    ]


_P = c_void_p
_SIGNATURES = {
    "spsim_b200_status_string": (c_char_p, [c_int]),
    "spsim_b200_last_error": (c_char_p, []),
    "spsim_b200_version": (c_char_p, []),
    "spsim_b200_init": (c_int, [c_int]),
    "spsim_b200_device_count": (c_int, [POINTER(c_int)]),
    "spsim_b200_molecule_create": (c_int, [c_int, _P, _P, _P, _P, c_int, _P, POINTER(c_void_p)]),
    "spsim_b200_molecule_create_f64": (c_int, [c_int, _P, _P, _P, _P, c_int, _P, POINTER(c_void_p)]),
    "spsim_b200_molecule_update_device": (c_int, [_P, _P, c_int, _P, _P, _P]),
    "spsim_b200_molecule_natoms": (c_int, [_P, POINTER(c_int)]),
    "spsim_b200_molecule_destroy": (c_int, [_P]),
    "spsim_b200_qset_from_list": (c_int, [c_int64, _P, c_int, POINTER(c_void_p)]),
    "spsim_b200_qset_from_detector": (
        c_int, [c_int, c_int, c_float, c_float, c_float, c_float, c_float, c_float, c_int, POINTER(c_void_p)]),
    "spsim_b200_qset_npix": (c_int, [_P, POINTER(c_int64)]),
    "spsim_b200_qset_copy_q": (c_int, [_P, _P]),
    "spsim_b200_qset_destroy": (c_int, [_P]),
    "spsim_b200_forward": (c_int, [_P, _P, _P, c_float, c_int, _P, _P, _P]),
    "spsim_b200_forward_batch": (c_int, [c_int, _P, _P, _P, c_float, c_int, _P, _P, _P]),
    "spsim_b200_structure_factor_host": (
        c_int, [c_int, _P, _P, _P, _P, c_float, c_int, _P, c_int64, _P, c_int, _P, _P]),
    "spsim_b200_structure_factor_host_spectrum": (
        c_int, [c_int, _P, _P, _P, _P, c_float, c_int, _P, c_float, c_float, c_int, c_int64, _P, c_int, _P, _P]),
    "spsim_b200_forward_spectrum": (c_int, [_P, _P, _P, c_float, c_int, c_float, c_float, c_int, _P, _P, _P]),
    "spsim_b200_forward_nufft": (c_int, [_P, _P, _P, c_float, c_double, _P, _P, _P]),
    "spsim_b200_forward_nufft_batch": (c_int, [_P, _P, c_int, _P, c_float, c_double, _P, _P, _P]),
    "spsim_b200_last_nufft_grid": (c_int, [POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
    "spsim_b200_set_nufft_interp": (c_int, [c_int]),
    "spsim_b200_structure_factor_host_nufft": (
        c_int, [c_int, _P, _P, c_float, c_int, c_int64, _P, c_double, _P, _P]),
    "spsim_b200_adjoint": (c_int, [_P, _P, c_int, _P, c_float, c_int, _P, _P, _P, _P, _P, _P]),
    "spsim_b200_detector_chain": (c_int, [POINTER(ChainParams), _P, POINTER(ChainOutputs), _P]),
    "spsim_b200_thomson": (c_int, [POINTER(ChainParams), _P, _P]),
    "spsim_b200_solid_angle": (c_int, [POINTER(ChainParams), _P, _P]),
    "spsim_b200_poisson": (c_int, [c_int64, _P, c_uint64, c_uint32, _P, _P]),
    "spsim_b200_photons": (c_int, [c_int64, _P, _P, _P, c_float, _P, _P]),
    "spsim_b200_photon_counts": (c_int, [POINTER(ChainParams), _P, _P, _P]),
    "spsim_b200_electrons": (c_int, [POINTER(ChainParams), _P, _P, _P]),
    "spsim_b200_binned_outputs": (c_int, [POINTER(ChainParams), _P, _P, _P, _P, _P]),
    "spsim_b200_hkl_for_detector": (
        c_int, [c_int, c_int, c_float, c_float, c_float, c_float, c_float, c_float, c_int, _P, _P]),
    "spsim_b200_synchronize": (c_int, [_P]),
    "spsim_b200_debug_stall_first_copy": (c_int, [c_int]),
    "spsim_b200_structure_factor_host_noalloc": (
        c_int, [c_int, _P, _P, _P, _P, c_float, c_int, _P, c_int64, _P, c_int, _P, _P]),
    "spsim_b200_timing_enable": (c_int, [c_int]),
    "spsim_b200_timing_read": (c_int, [POINTER(c_double), c_int, POINTER(c_int)]),
    "spsim_b200_last_forward_stats": (c_int, [POINTER(c_double), POINTER(c_double)]),
    "spsim_b200_set_variant": (c_int, [c_int, c_int, c_int]),
    "spsim_b200_last_variant": (c_int, [POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
    "spsim_b200_last_phase_word": (c_int, [POINTER(c_int)]),
    "spsim_b200_last_pair_narrow": (c_int, [POINTER(c_int)]),
    "spsim_b200_release_scratch": (None, []),
    "spsim_b200_autotune": (c_int, [_P, _P, c_int, _P, POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
    "spsim_b200_autotune_batch": (c_int, [c_int, _P, _P, _P, c_int, _P, POINTER(c_int), POINTER(c_int),
                                          POINTER(c_int)]),
    "spsim_b200_clear_tuning": (c_int, []),
    "spsim_b200_set_legacy_precision": (None, [c_int]),
    "spsim_b200_set_legacy_nufft_eps": (None, [c_double]),
    "spsim_b200_get_legacy_nufft_eps": (c_double, []),
    "spsim_b200_get_legacy_precision": (c_int, []),
    "spsim_b200_set_noise_seed": (None, [c_uint64]),
    "spsim_b200_set_shot_chunks": (None, [c_int]),
    "spsim_b200_get_shot_chunks": (c_int, []),
}

_lock = threading.Lock()
_lib = None


def lib():
    """The loaded library (built in-tree by spsim_b200.build)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise ImportError(
                        "libspsim_b200.so not found at %s; build it with `python -m spsim_b200.build`" % LIB_PATH)
                L = ctypes.CDLL(LIB_PATH)
                for name, (res, args) in _SIGNATURES.items():
                    f = getattr(L, name)
                    f.restype = res
                    f.argtypes = args
                _lib = L
    return _lib


def check(status):
    """Raise SpsimError for a non-zero status."""
    if status != SPSIM_OK:
        raise SpsimError(status, lib().spsim_b200_last_error().decode(errors="replace"))


_device_state = threading.local()


def use_device(index):
    """Make `index` the native library's current CUDA device on this thread.

    The library links its own CUDA runtime, whose current-device state is
    separate from PyTorch's, so every entry point that allocates or launches
    goes through here first."""
    if getattr(_device_state, "dev", None) != index:
        check(lib().spsim_b200_init(int(index)))
        _device_state.dev = index


def device_count():
    n = c_int(0)
    check(lib().spsim_b200_device_count(ctypes.byref(n)))
    return n.value


def version():
    return lib().spsim_b200_version().decode()
