"""Drop-in for spsim's SWIG module ``spsim_pybackend`` (src/spsim_pybackend.i).

The SWIG module wraps spsim.h, config.h, diffraction.h and molecule.h
(src/spsim_pybackend.i:140-146) so Python code calls the C functions by name
and reads struct fields as attributes.  This module exposes the same names
from libspsim_b200.so through ctypes: the structs are ctypes Structures with
the reference layouts (include/spsim_types.h), the functions take and return
pointers to them, and array fields are reachable as numpy views through
``as_array``.

    opts = set_defaults(); read_options_file("spsim.conf", opts)
    mol = get_molecule_from_atoms(Z, pos)          # spsim_b200.spsim helper
    pat = simulate_shot(mol, opts)
    I = as_array(pat.contents.ints, opts.contents.detector.contents.nx * ...)
"""
import ctypes
from ctypes import POINTER, c_char, c_char_p, c_float, c_int, c_void_p

import numpy as np

from . import _native


class Complex(ctypes.Structure):
    _fields_ = [("re", c_float), ("im", c_float)]


class SpRotation(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_uint), ("cols", ctypes.c_uint), ("data", POINTER(c_float))]


class Chem_Formula(ctypes.Structure):
    _fields_ = [("n_elements", c_int), ("atomic_number", POINTER(c_int)), ("quantity", POINTER(c_int))]


class Molecule(ctypes.Structure):
    _fields_ = [("natoms", c_int), ("atomic_number", POINTER(c_int)), ("pos", POINTER(c_float)),
                ("delta_atoms", c_int)]


class Experiment(ctypes.Structure):
    _fields_ = [(n, c_float) for n in ("wavelength", "bandwidth", "exposure_time", "beam_intensity",
                                       "beam_center_x", "beam_center_y", "beam_fwhm", "beam_energy",
                                       "photon_energy", "focal_diameter")] + [("polarization", c_int)]


CCD_ARRAYS = ("photons_per_pixel", "thomson_correction", "solid_angle", "photon_count", "electrons_per_pixel",
              "real_output", "noiseless_output")


class CCD(ctypes.Structure):
    _fields_ = [(n, POINTER(c_float)) for n in CCD_ARRAYS] + \
               [(n, c_float) for n in ("distance", "width", "height", "depth", "pixel_width", "pixel_height",
                                       "pixel_depth", "quantum_efficiency", "electron_hole_production_energy",
                                       "readout_noise", "dark_current", "linear_full_well")] + \
               [(n, c_int) for n in ("binning_x", "binning_y", "binning_z", "nx", "ny", "nz")] + \
               [("maximum_value", c_float), ("spherical", c_int), ("gaussian_blurring", c_float),
                ("real_space_blurring", c_float), ("center_x", c_float), ("center_y", c_float),
                ("center_z", c_float), ("n_patterns", c_int)]


class Options(ctypes.Structure):
    _fields_ = [("input_type", c_int), ("chem_formula", POINTER(Chem_Formula)),
                ("experiment", POINTER(Experiment)), ("detector", POINTER(CCD)),
                ("pdb_filename", c_char * 1024), ("sf_filename", c_char * 1024),
                ("hkl_grid_filename", c_char * 1024), ("box_type", c_int), ("box_dimension", c_float),
                ("use_fft_for_sf", c_int), ("use_nfft_for_sf", c_int), ("b_factor", c_float),
                ("origin_to_com", c_int), ("euler_orientation", c_float * 3), ("random_orientation", c_int),
                ("n_patterns", c_int), ("vectorize", c_int), ("delta_atoms", c_int), ("fast_exit", c_int),
                ("crystal_size", c_int * 3), ("crystal_cell", c_float * 6)] + \
               [(n, c_int) for n in ("use_cuda", "wavelength_samples", "random_seed", "output_sf_vtk",
                                     "output_scatt_int", "output_ewald_vtk", "output_intensities",
                                     "output_noiseless_photons", "output_photons", "output_electron_pixel_vtk",
                                     "output_noiseless_count", "output_count", "output_realspace_histogram",
                                     "output_scattering_factors", "output_solid_angles", "output_real_space",
                                     "verbosity_level")]


class Diffraction_Pattern(ctypes.Structure):
    _fields_ = [("ints", POINTER(c_float)), ("F", POINTER(Complex)), ("N_pix", c_int), ("max_s", c_float * 3),
                ("d_s", c_float * 3), ("HKL_list", POINTER(c_float)), ("HKL_list_size", c_int),
                ("rot", POINTER(SpRotation))]


P = POINTER
_PROTOS = {
    "set_defaults": (P(Options), []),
    "read_options_file": (None, [c_char_p, P(Options)]),
    "write_options_file": (None, [c_char_p, P(Options)]),
    "get_HKL_list_for_detector": (P(c_float), [P(CCD), P(Experiment), P(c_int)]),
    "get_HKL_list_for_3d_detector": (P(c_float), [P(CCD), P(Experiment), P(c_int)]),
    "apply_orientation_to_HKL_list": (P(SpRotation), [P(P(c_float)), P(c_int), P(Options)]),
    "get_HKL_list": (P(c_float), [P(Options), P(c_int)]),
    "compute_pattern_on_list": (P(Diffraction_Pattern), [P(Molecule), P(c_float), c_int, c_float, P(Experiment),
                                                         P(Options)]),
    "vector_compute_pattern_on_list": (P(Diffraction_Pattern), [P(Molecule), P(c_float), c_int, c_float,
                                                                P(Experiment), P(Options)]),
    "cuda_compute_pattern_on_list": (P(Diffraction_Pattern), [P(Molecule), P(c_float), c_int, c_float,
                                                              P(Experiment), P(Options)]),
    "cuda_compute_pattern_on_list2": (P(Diffraction_Pattern), [P(Molecule), P(c_float), c_int, c_float,
                                                               P(Experiment), P(Options)]),
    "compute_pattern_on_list_by_nfft": (P(Diffraction_Pattern), [P(Molecule), P(c_float), c_int, P(CCD), c_float,
                                                                 P(Options)]),
    "compute_sf": (P(Diffraction_Pattern), [P(Molecule), P(c_float), c_int, P(Options)]),
    "calculate_thomson_correction": (None, [P(CCD), P(Experiment)]),
    "calculate_pixel_solid_angle": (None, [P(CCD)]),
    "calculate_photons_per_pixel": (None, [P(Diffraction_Pattern), P(Options)]),
    "generate_poisson_noise": (None, [P(CCD)]),
    "calculate_electrons_per_pixel": (None, [P(CCD), P(Experiment)]),
    "calculate_real_detector_output": (None, [P(CCD), P(Experiment)]),
    "calculate_noiseless_detector_output": (None, [P(CCD), P(Experiment)]),
    "simulate_shot": (P(Diffraction_Pattern), [P(Molecule), P(Options)]),
    "free_stuff": (None, [P(Diffraction_Pattern), P(Options)]),
    "free_diffraction_pattern": (None, [P(Diffraction_Pattern)]),
    "free_output_in_options": (None, [P(Options)]),
    "alloc_mol": (P(Molecule), []),
    "add_atom_to_mol": (None, [P(Molecule), c_int, c_float, c_float, c_float]),
    "free_mol": (None, [P(Molecule)]),
    "get_Molecule_from_pdb": (P(Molecule), [c_char_p]),
    "crystal_axis_to_cartesian": (None, [P(Options), c_int, P(c_float), P(c_float), P(c_float)]),
    "crystal_cell_matrix": (None, [P(Options), P(c_float)]),
    "calculate_pattern_from_crystal": (None, [P(c_float), P(Complex), P(c_float), c_int, P(Options)]),
    "get_Molecule_from_formula": (P(Molecule), [P(Chem_Formula), P(Options)]),
    "write_pdb_from_mol": (None, [c_char_p, P(Molecule)]),
    "origin_to_center_of_mass": (None, [P(Molecule)]),
    "get_molecule": (P(Molecule), [P(Options)]),
    "write_2D_array_to_vtk": (None, [P(c_float), c_int, c_int, c_char_p]),
    "write_3D_array_to_vtk": (None, [P(c_float), c_int, c_int, c_int, c_char_p]),
    "get_my_loop_start_and_end": (None, [c_int, P(c_int), P(c_int)]),
    "syncronize_patterns": (None, [P(Diffraction_Pattern)]),
    "sum_patterns": (None, [P(Diffraction_Pattern)]),
    "output_array": (None, [c_char_p, c_int, P(c_float), P(SpRotation), P(Options)]),
    "output_carray": (None, [c_char_p, c_int, P(Complex), P(SpRotation), P(Options)]),
    "output_files": (None, [P(Diffraction_Pattern), P(Options), c_int]),
}

_bound = {}


def _fn(name):
    f = _bound.get(name)
    if f is None:
        f = getattr(_native.lib(), name)
        res, args = _PROTOS[name]
        f.restype = res
        f.argtypes = args
        _bound[name] = f
    return f


def _path(s):
    return s.encode() if isinstance(s, str) else s


def _gpu_call(name, *args):
    """Reference-shaped calls that launch kernels: make sure the library's
    device matches PyTorch's current one when PyTorch is in use."""
    try:
        import torch

        if torch.cuda.is_available():
            _native.use_device(torch.cuda.current_device())
    except ImportError:
        pass
    return _fn(name)(*args)


# ---- configuration
def set_defaults():
    return _fn("set_defaults")()


def read_options_file(filename, opts):
    _fn("read_options_file")(_path(filename), opts)


def write_options_file(filename, opts):
    _fn("write_options_file")(_path(filename), opts)


# ---- geometry
def get_HKL_list_for_detector(det, exp, size):
    return _gpu_call("get_HKL_list_for_detector", det, exp, size)


def get_HKL_list_for_3d_detector(det, exp, size):
    return _gpu_call("get_HKL_list_for_3d_detector", det, exp, size)


def apply_orientation_to_HKL_list(hkl_ptr_ptr, size, opts):
    return _fn("apply_orientation_to_HKL_list")(hkl_ptr_ptr, size, opts)


def get_HKL_list(opts, size):
    return _gpu_call("get_HKL_list", opts, size)


# ---- structure factor
def compute_pattern_on_list(mol, HKL_list, HKL_list_size, B, exp, opts):
    return _gpu_call("compute_pattern_on_list", mol, _floats(HKL_list), HKL_list_size, B, exp, opts)


def vector_compute_pattern_on_list(mol, HKL_list, HKL_list_size, B, exp, opts):
    return _gpu_call("vector_compute_pattern_on_list", mol, _floats(HKL_list), HKL_list_size, B, exp, opts)


def cuda_compute_pattern_on_list(mol, HKL_list, HKL_list_size, B, exp, opts):
    return _gpu_call("cuda_compute_pattern_on_list", mol, _floats(HKL_list), HKL_list_size, B, exp, opts)


def cuda_compute_pattern_on_list2(mol, HKL_list, HKL_list_size, B, exp, opts):
    return _gpu_call("cuda_compute_pattern_on_list2", mol, _floats(HKL_list), HKL_list_size, B, exp, opts)


def compute_pattern_on_list_by_nfft(mol, HKL_list, HKL_list_size, det, B, opts):
    return _gpu_call("compute_pattern_on_list_by_nfft", mol, _floats(HKL_list), HKL_list_size, det, B, opts)


def compute_sf(mol, HKL_list, HKL_list_size, opts):
    return _gpu_call("compute_sf", mol, _floats(HKL_list), HKL_list_size, opts)


# ---- detector chain
def calculate_thomson_correction(det, exp):
    _gpu_call("calculate_thomson_correction", det, exp)


def calculate_pixel_solid_angle(det):
    _gpu_call("calculate_pixel_solid_angle", det)


def calculate_photons_per_pixel(pattern, opts):
    _gpu_call("calculate_photons_per_pixel", pattern, opts)


def generate_poisson_noise(det):
    _gpu_call("generate_poisson_noise", det)


def calculate_electrons_per_pixel(det, exp):
    _gpu_call("calculate_electrons_per_pixel", det, exp)


def calculate_real_detector_output(det, exp):
    _gpu_call("calculate_real_detector_output", det, exp)


def calculate_noiseless_detector_output(det, exp):
    _gpu_call("calculate_noiseless_detector_output", det, exp)


# ---- orchestration
def simulate_shot(mol, opts):
    return _gpu_call("simulate_shot", mol, opts)


def free_stuff(pattern, opts):
    _fn("free_stuff")(pattern, opts)


def free_diffraction_pattern(pattern):
    _fn("free_diffraction_pattern")(pattern)


def free_output_in_options(opts):
    _fn("free_output_in_options")(opts)


# ---- molecules
def alloc_mol():
    return _fn("alloc_mol")()


def add_atom_to_mol(mol, atomic_number, x, y, z):
    _fn("add_atom_to_mol")(mol, int(atomic_number), float(x), float(y), float(z))


def free_mol(mol):
    _fn("free_mol")(mol)


# ---- output files (src/spsim.c:146-279): <basename>-NNNNN.cxi
def output_array(basename, index, array, rot, opts):
    """array: a float32 numpy array of the detector's pixels (or a ctypes float pointer)."""
    keep = np.ascontiguousarray(array, np.float32) if isinstance(array, np.ndarray) else None
    ptr = keep.ctypes.data_as(P(c_float)) if keep is not None else array
    _fn("output_array")(_path(basename), int(index), ptr, rot, opts)


def output_carray(basename, index, array, rot, opts):
    """array: a complex64 numpy array (or a ctypes Complex pointer)."""
    keep = np.ascontiguousarray(array, np.complex64) if isinstance(array, np.ndarray) else None
    ptr = keep.ctypes.data_as(P(Complex)) if keep is not None else array
    _fn("output_carray")(_path(basename), int(index), ptr, rot, opts)


def output_files(pattern, opts, index):
    _fn("output_files")(pattern, opts, int(index))


# ---- distribution (single-process semantics)
def get_my_loop_start_and_end(size):
    s, e = c_int(0), c_int(0)
    _fn("get_my_loop_start_and_end")(int(size), ctypes.byref(s), ctypes.byref(e))
    return s.value, e.value


def syncronize_patterns(pat):
    _fn("syncronize_patterns")(pat)


def sum_patterns(pat):
    _fn("sum_patterns")(pat)


# ---- helpers
def set_precision(precision):
    """Precision of the reference-shaped structure-factor calls: "f32", "f32_fast" or "fp64"."""
    _native.lib().spsim_b200_set_legacy_precision(_native.PRECISIONS.get(precision, precision))


def set_noise_seed(seed):
    _native.lib().spsim_b200_set_noise_seed(int(seed))


def set_nufft_eps(eps):
    """Relative error of the NUFFT structure factor behind compute_pattern_on_list_by_nfft
    and use_nfft_for_sf (default 1e-8)."""
    _native.lib().spsim_b200_set_legacy_nufft_eps(float(eps))


def get_nufft_eps():
    return _native.lib().spsim_b200_get_legacy_nufft_eps()


def set_shot_chunks(chunks):
    """Row chunks of simulate_shot (0: automatic, 1: none; see spsim_b200_set_shot_chunks)."""
    _native.lib().spsim_b200_set_shot_chunks(int(chunks))


def get_shot_chunks():
    return _native.lib().spsim_b200_get_shot_chunks()


def _floats(a):
    if isinstance(a, np.ndarray):
        a = np.ascontiguousarray(a, np.float32)
        ptr = a.ctypes.data_as(POINTER(c_float))
        ptr._keep = a  # keep the array alive for the call
        return ptr
    return a


def as_array(ptr, n, dtype=np.float32):
    """A numpy copy of n elements behind a ctypes pointer (float arrays, Complex arrays)."""
    if isinstance(ptr, ctypes.POINTER(Complex)) or getattr(ptr, "_type_", None) is Complex:
        raw = np.ctypeslib.as_array(ctypes.cast(ptr, POINTER(c_float)), shape=(2 * n,)).copy()
        return raw[0::2] + 1j * raw[1::2]
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


# ---- molecule files and VTK output (src/molecule.c, src/io.c)
def get_Molecule_from_pdb(filename):
    return _fn("get_Molecule_from_pdb")(_path(filename))


def get_Molecule_from_formula(form, opts):
    return _fn("get_Molecule_from_formula")(form, opts)


def write_pdb_from_mol(filename, mol):
    _fn("write_pdb_from_mol")(_path(filename), mol)


def origin_to_center_of_mass(mol):
    _fn("origin_to_center_of_mass")(mol)


def get_molecule(opts):
    return _fn("get_molecule")(opts)


def write_2D_array_to_vtk(F, nx, ny, filename):
    _fn("write_2D_array_to_vtk")(_floats(F), int(nx), int(ny), _path(filename))


def write_3D_array_to_vtk(F, nx, ny, nz, filename):
    _fn("write_3D_array_to_vtk")(_floats(F), int(nx), int(ny), int(nz), _path(filename))


# ---- crystal lattice (src/crystal.c)
CrystalA, CrystalB, CrystalC = 0, 1, 2


def crystal_axis_to_cartesian(opts, axis, x, y, z):
    _fn("crystal_axis_to_cartesian")(opts, int(axis), x, y, z)


def crystal_cell_matrix(opts, matrix):
    _fn("crystal_cell_matrix")(opts, _floats(matrix))


def calculate_pattern_from_crystal(I, F, HKL_list, HKL_list_size, opts):
    _gpu_call("calculate_pattern_from_crystal", I, F, _floats(HKL_list), int(HKL_list_size), opts)
