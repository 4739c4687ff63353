"""ORACLE — test infrastructure only.

ctypes access to the checkers built by oracle/Makefile:
  * oracle/_build/libspsim_oracle.so : the FP64 restatement (sf_oracle.c)
  * oracle/_ref/libspsim_ref.so      : spsim's own CPU sources compiled unchanged
  * oracle/_ref/libspsim_refgpu.so   : spsim's own CUDA source compiled unchanged
                                       (GPU comparison point, GPU tests only)
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product never does.
"""
import ctypes
import os
from ctypes import POINTER, c_char, c_double, c_float, c_int, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "libspsim_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libspsim_ref.so")
REF_GPU_LIB = os.path.join(HERE, "_ref", "libspsim_refgpu.so")

_oracle = None
_ref = None


def _p(a):
    return a.ctypes.data_as(c_void_p) if a is not None else None


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_LIB):
            raise ImportError("oracle not built: make -C oracle oracle")
        _oracle = ctypes.CDLL(ORACLE_LIB)
        _oracle.oracle_scatt_factor.restype = c_double
        _oracle.oracle_scatt_factor.argtypes = [c_double, c_int, c_double]
    return _oracle


def ref_available():
    return os.path.exists(REF_LIB)


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise ImportError("reference library not built: make -C oracle ref REF=<spsim tree>")
        _ref = ctypes.CDLL(REF_LIB)
    return _ref


# ---------------------------------------------------------------- FP64 oracle

def scatt_factor(q_len, Z, B=0.0):
    return oracle_lib().oracle_scatt_factor(float(q_len), int(Z), float(B))


def atomsf_table():
    """The oracle's coefficient table in use: float32 (100, 9), rows a1..a4, b1..b4, c."""
    L = oracle_lib()
    L.oracle_get_atomsf_row.argtypes = [c_int, c_void_p]
    out = np.zeros((100, 9), np.float32)
    for z in range(100):
        L.oracle_get_atomsf_row(z, _p(out[z]))
    return out


def set_atomsf_table(table):
    """Replace every row of the oracle's coefficient table."""
    L = oracle_lib()
    L.oracle_set_atomsf_row.argtypes = [c_int, c_void_p]
    t = np.ascontiguousarray(table, np.float32).reshape(100, 9)
    for z in range(100):
        L.oracle_set_atomsf_row(z, _p(t[z]))


def reset_atomsf_table():
    """Back to the compiled-in table."""
    oracle_lib().oracle_reset_atomsf()


def atomsf_lib_table(path, base=None):
    """The coefficient table spsim uses when ./atomsf.lib exists
    (src/diffraction.c:118-177, fill_ff_tables): starting from the compiled-in
    table, every row's a1 is set to -1; after the leading comment lines (those
    starting with "AD") the file holds 5-line records: a name line; a line with
    Z (read by %d from its start) and c (read by %f from column 24 on); a1..a4
    and b1..b4 in 16-column fields on the next two lines; one more line.  A
    record replaces row Z only the first time Z appears (a1 still -1)."""
    t = np.array(atomsf_table() if base is None else base, np.float32)
    t[:, 0] = -1.0
    lines = open(path).read().splitlines(keepends=True)
    i = 0
    while i < len(lines) and lines[i].startswith("AD"):
        i += 1

    def num(s, conv):
        tok = s.split()
        try:
            return conv(tok[0]) if tok else None
        except ValueError:
            return None

    while i < len(lines):  # lines[i]: the record's name line (a blank line counts)
        if i + 3 >= len(lines):
            break
        zl, al, bl = lines[i + 1], lines[i + 2], lines[i + 3]
        z = num(zl, int)
        if z is None or not 0 <= z < 100:
            break
        if t[z, 0] == -1.0:
            c = num(zl[23:], float)
            if c is not None:
                t[z, 8] = c
            for k in range(4):
                a, b = num(al[16 * k:], float), num(bl[16 * k:], float)
                if a is not None:
                    t[z, k] = a
                if b is not None:
                    t[z, 4 + k] = b
        i += 5
    return t


def hkl_detector(nx, ny, width, height, distance, wavelength, center_x=0.0, center_y=0.0, spherical=False):
    q = np.empty((nx * ny, 3), np.float64)
    L = oracle_lib()
    L.oracle_hkl_detector.argtypes = [c_int, c_int, c_float, c_float, c_float, c_float, c_float, c_float, c_int,
                                      c_void_p]
    L.oracle_hkl_detector(nx, ny, width, height, distance, center_x, center_y, wavelength, int(spherical), _p(q))
    return q


def structure_factor(Z, pos, q, occ=None, bfac=None, B=0.0, delta_atoms=False, beam=None, nthreads=None):
    """FP64 F (complex128) and I = |F|^2 (float64) for atoms (Z, pos [m]) at q [1/m]."""
    Z = np.ascontiguousarray(Z, np.int32)
    pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
    q = np.ascontiguousarray(q, np.float64).reshape(-1, 3)
    occ = np.ascontiguousarray(occ, np.float64) if occ is not None else None
    bfac = np.ascontiguousarray(bfac, np.float64) if bfac is not None else None
    n = q.shape[0]
    fr, fi, I = np.empty(n), np.empty(n), np.empty(n)
    beam = (0.0, 0.0, 0.0) if beam is None else tuple(float(b) for b in beam)
    L = oracle_lib()
    L.oracle_structure_factor.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_int, c_double,
                                          c_double, c_double, ctypes.c_long, c_void_p, c_void_p, c_void_p, c_void_p,
                                          c_int]
    L.oracle_structure_factor(len(Z), _p(Z), _p(pos), _p(occ), _p(bfac), float(B), int(delta_atoms), float(beam[0]),
                              float(beam[1]), float(beam[2]), n, _p(q), _p(fr), _p(fi), _p(I),
                              int(nthreads or os.cpu_count() or 1))
    return fr + 1j * fi, I


def structure_factor_spectrum(Z, pos, q, wavelength, bandwidth, samples, occ=None, bfac=None, B=0.0,
                              delta_atoms=False, beam=None, nthreads=None):
    """FP64 polychromatic structure factor (spsim's spectrum kernel semantics,
    src/diffraction.cu:415-476): (F complex128, I float64)."""
    L = oracle_lib()
    Z = np.ascontiguousarray(Z, np.int32)
    pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
    q = np.ascontiguousarray(q, np.float64).reshape(-1, 3)
    occ = np.ascontiguousarray(occ, np.float64) if occ is not None else None
    bfac = np.ascontiguousarray(bfac, np.float64) if bfac is not None else None
    beam = (0.0, 0.0, 0.0) if beam is None else tuple(float(b) for b in beam)
    n = q.shape[0]
    Fr, Fi, I = np.zeros(n), np.zeros(n), np.zeros(n)
    L.oracle_structure_factor_spectrum.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_int,
                                                   c_double, c_double, c_double, c_double, c_double, c_int,
                                                   ctypes.c_long, c_void_p, c_void_p, c_void_p, c_void_p, c_int]
    L.oracle_structure_factor_spectrum(len(Z), _p(Z), _p(pos), _p(occ), _p(bfac), float(B), int(delta_atoms),
                                       float(beam[0]), float(beam[1]), float(beam[2]), float(wavelength),
                                       float(bandwidth), int(samples), n, _p(q), _p(Fr), _p(Fi), _p(I),
                                       nthreads or os.cpu_count() or 1)
    return Fr + 1j * Fi, I


def structure_factor_vjp(Z, pos, q, g, occ=None, bfac=None, nthreads=None):
    """FP64 dL/dpos (N,3), dL/docc (N,), dL/dB (N,) for dL/dI = g."""
    Z = np.ascontiguousarray(Z, np.int32)
    pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
    q = np.ascontiguousarray(q, np.float64).reshape(-1, 3)
    g = np.ascontiguousarray(g, np.float64).reshape(-1)
    occ = np.ascontiguousarray(occ, np.float64) if occ is not None else None
    bfac = np.ascontiguousarray(bfac, np.float64) if bfac is not None else None
    N = len(Z)
    dp, do, db = np.empty((N, 3)), np.empty(N), np.empty(N)
    L = oracle_lib()
    L.oracle_structure_factor_vjp.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_long, c_void_p,
                                              c_void_p, c_void_p, c_void_p, c_void_p, c_int]
    L.oracle_structure_factor_vjp(N, _p(Z), _p(pos), _p(occ), _p(bfac), q.shape[0], _p(q), _p(g), _p(dp), _p(do),
                                  _p(db), int(nthreads or os.cpu_count() or 1))
    return dp, do, db


def thomson(nx, ny, width, height, distance, polarization=0, center_x=0.0, center_y=0.0, nz=1):
    out = np.empty(nx * ny * nz)
    L = oracle_lib()
    L.oracle_thomson.argtypes = [c_int, c_int, c_int, c_float, c_float, c_float, c_float, c_float, c_int, c_void_p]
    L.oracle_thomson(nx, ny, nz, width, height, distance, center_x, center_y, polarization, _p(out))
    return out


def solid_angle(nx, ny, width, height, distance, pixel_width, pixel_height, spherical=False, center_x=0.0,
                center_y=0.0, nz=1):
    out = np.empty(nx * ny * nz)
    L = oracle_lib()
    L.oracle_solid_angle.argtypes = [c_int, c_int, c_int, c_float, c_float, c_float, c_float, c_float, c_float,
                                     c_float, c_int, c_void_p]
    L.oracle_solid_angle(nx, ny, nz, width, height, distance, center_x, center_y, pixel_width, pixel_height,
                         int(spherical), _p(out))
    return out


def noiseless_output(photons, nx, ny, bx, by, qe, wavelength, e_hole, full_well, max_value, nz=1, bz=1):
    photons = np.ascontiguousarray(photons, np.float64)
    out = np.empty((nx // bx) * (ny // by) * (nz // bz))
    L = oracle_lib()
    L.oracle_noiseless_output.argtypes = [c_int] * 6 + [c_void_p] + [c_double] * 5 + [c_void_p]
    L.oracle_noiseless_output(nx, ny, nz, bx, by, bz, _p(photons), qe, wavelength, e_hole, full_well, max_value,
                              _p(out))
    return out


def real_output(electrons, noise, nx, ny, bx, by, dark, exposure, full_well, max_value, clamp=False, nz=1, bz=1):
    electrons = np.ascontiguousarray(electrons, np.float64)
    noise = np.ascontiguousarray(noise, np.float64) if noise is not None else None
    out = np.empty((nx // bx) * (ny // by) * (nz // bz))
    L = oracle_lib()
    L.oracle_real_output.argtypes = [c_int] * 6 + [c_void_p, c_double, c_double, c_void_p, c_double, c_double, c_int,
                                                   c_void_p]
    L.oracle_real_output(nx, ny, nz, bx, by, bz, _p(electrons), dark, exposure, _p(noise), full_well, max_value,
                         int(clamp), _p(out))
    return out


def philox(c0, c1, c2, c3, seed):
    out = np.empty(4, np.uint32)
    L = oracle_lib()
    L.oracle_philox.argtypes = [c_uint32] * 4 + [c_uint64, c_void_p]
    L.oracle_philox(c0, c1, c2, c3, seed, _p(out))
    return out


def poisson(lam, seed, pattern=0):
    lam = np.ascontiguousarray(lam, np.float32)
    out = np.empty_like(lam)
    L = oracle_lib()
    L.oracle_poisson.argtypes = [ctypes.c_long, c_void_p, c_uint32, c_uint64, c_void_p]
    L.oracle_poisson(lam.size, _p(lam), pattern, seed, _p(out))
    return out


def readout_noise(n, sigma, seed, pattern=0):
    out = np.empty(n, np.float32)
    L = oracle_lib()
    L.oracle_readout_noise.argtypes = [ctypes.c_long, c_float, c_uint32, c_uint64, c_void_p]
    L.oracle_readout_noise(n, sigma, pattern, seed, _p(out))
    return out


# ---------------------------------------------------------------- reference (spsim's own C)

class RefComplex(ctypes.Structure):
    _fields_ = [("re", c_float), ("im", c_float)]


class RefMolecule(ctypes.Structure):  # include/config.h:50-58
    _fields_ = [("natoms", c_int), ("atomic_number", POINTER(c_int)), ("pos", POINTER(c_float)),
                ("delta_atoms", c_int)]


class RefExperiment(ctypes.Structure):  # include/config.h:60-76
    _fields_ = [(n, c_float) for n in ("wavelength", "bandwidth", "exposure_time", "beam_intensity", "beam_center_x",
                                       "beam_center_y", "beam_fwhm", "beam_energy", "photon_energy",
                                       "focal_diameter")] + [("polarization", c_int)]


class RefCCD(ctypes.Structure):  # include/config.h:78-128
    _fields_ = [(n, POINTER(c_float)) for n in ("photons_per_pixel", "thomson_correction", "solid_angle",
                                                "photon_count", "electrons_per_pixel", "real_output",
                                                "noiseless_output")] + \
               [(n, c_float) for n in ("distance", "width", "height", "depth", "pixel_width", "pixel_height",
                                       "pixel_depth", "quantum_efficiency", "electron_hole_production_energy",
                                       "readout_noise", "dark_current", "linear_full_well")] + \
               [(n, c_int) for n in ("binning_x", "binning_y", "binning_z", "nx", "ny", "nz")] + \
               [("maximum_value", c_float), ("spherical", c_int), ("gaussian_blurring", c_float),
                ("real_space_blurring", c_float), ("center_x", c_float), ("center_y", c_float),
                ("center_z", c_float), ("n_patterns", c_int)]


class RefChemFormula(ctypes.Structure):
    _fields_ = [("n_elements", c_int), ("atomic_number", POINTER(c_int)), ("quantity", POINTER(c_int))]


class RefOptions(ctypes.Structure):  # include/config.h:131-181
    _fields_ = [("input_type", c_int), ("chem_formula", POINTER(RefChemFormula)),
                ("experiment", POINTER(RefExperiment)), ("detector", POINTER(RefCCD)),
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


class RefPattern(ctypes.Structure):  # include/diffraction.h:46-62
    _fields_ = [("ints", POINTER(c_float)), ("F", POINTER(RefComplex)), ("N_pix", c_int), ("max_s", c_float * 3),
                ("d_s", c_float * 3), ("HKL_list", POINTER(c_float)), ("HKL_list_size", c_int),
                ("rot", c_void_p)]


def _ref_setup():
    L = ref_lib()
    for name in ("compute_pattern_on_list", "vector_compute_pattern_on_list"):
        f = getattr(L, name)
        f.restype = POINTER(RefPattern)
        f.argtypes = [POINTER(RefMolecule), c_void_p, c_int, c_float, POINTER(RefExperiment), POINTER(RefOptions)]
    L.set_defaults.restype = POINTER(RefOptions)
    L.get_HKL_list_for_detector.restype = POINTER(c_float)
    L.get_HKL_list_for_detector.argtypes = [POINTER(RefCCD), POINTER(RefExperiment), POINTER(c_int)]
    return L


def ref_defaults():
    L = _ref_setup()
    return L.set_defaults()


def ref_hkl_detector(nx, ny, width, height, distance, wavelength, center_x=0.0, center_y=0.0, spherical=False):
    L = _ref_setup()
    det = RefCCD(nx=nx, ny=ny, nz=1, width=width, height=height, distance=distance, center_x=center_x,
                 center_y=center_y, spherical=int(spherical))
    exp = RefExperiment(wavelength=wavelength)
    n = c_int(0)
    p = L.get_HKL_list_for_detector(ctypes.byref(det), ctypes.byref(exp), ctypes.byref(n))
    out = np.ctypeslib.as_array(p, shape=(n.value * 3,)).copy().reshape(-1, 3)
    ctypes.CDLL(None).free(ctypes.cast(p, c_void_p))
    return out


def ref_pattern(Z, pos, hkl, B=0.0, vector=False, delta_atoms=False, beam=None, verbosity=0, slab=None):
    """spsim's own compute_pattern_on_list / vector_compute_pattern_on_list (float F, ints).

    slab=(start, end) restricts the evaluation to a contiguous pixel range."""
    L = _ref_setup()
    Z = np.ascontiguousarray(Z, np.int32)
    pos = np.ascontiguousarray(pos, np.float32).reshape(-1)
    hkl = np.ascontiguousarray(hkl, np.float32).reshape(-1, 3)
    if slab is not None:
        hkl = np.ascontiguousarray(hkl[slab[0]:slab[1]])
    mol = RefMolecule(len(Z), Z.ctypes.data_as(POINTER(c_int)), pos.ctypes.data_as(POINTER(c_float)), 0)
    exp = RefExperiment()
    if beam is not None:
        exp.beam_fwhm, exp.beam_center_x, exp.beam_center_y = beam
    opts = RefOptions()
    opts.delta_atoms = int(delta_atoms)
    opts.verbosity_level = verbosity
    fn = L.vector_compute_pattern_on_list if vector else L.compute_pattern_on_list
    res = fn(ctypes.byref(mol), _p(hkl), hkl.shape[0], float(B), ctypes.byref(exp), ctypes.byref(opts))
    n = hkl.shape[0]
    Fr = np.ctypeslib.as_array(ctypes.cast(res.contents.F, POINTER(c_float)), shape=(2 * n,)).copy()
    I = np.ctypeslib.as_array(res.contents.ints, shape=(n,)).copy()
    libc = ctypes.CDLL(None)
    for ptr in (res.contents.F, res.contents.ints, res.contents.HKL_list):
        libc.free(ctypes.cast(ptr, c_void_p))
    libc.free(ctypes.cast(res, c_void_p))
    return Fr[0::2] + 1j * Fr[1::2], I


_refgpu = None


def ref_gpu_lib():
    """spsim's CUDA path (src/diffraction.cu) built for sm_100a, or None when absent."""
    global _refgpu
    if _refgpu is None and os.path.exists(REF_GPU_LIB):
        L = ctypes.CDLL(REF_GPU_LIB)
        for name in ("cuda_compute_pattern_on_list", "cuda_compute_pattern_on_list2"):
            f = getattr(L, name)
            f.restype = POINTER(RefPattern)
            f.argtypes = [POINTER(RefMolecule), c_void_p, c_int, c_float, POINTER(RefExperiment),
                          POINTER(RefOptions)]
        _refgpu = L
    return _refgpu


def ref_gpu_pattern(Z, pos, hkl, B=0.0, wavelength_samples=1, bandwidth=0.0, wavelength=0.0):
    """spsim's cuda_compute_pattern_on_list2 (src/diffraction.cu:235-339): float F and
    ints from CUDA_scattering_from_all_atoms (or the spectrum kernel when
    wavelength_samples > 1 and bandwidth > 0), 100 atoms per launch."""
    L = ref_gpu_lib()
    if L is None:
        raise FileNotFoundError(REF_GPU_LIB)
    Z = np.ascontiguousarray(Z, np.int32)
    pos = np.ascontiguousarray(pos, np.float32).reshape(-1)
    hkl = np.ascontiguousarray(hkl, np.float32).reshape(-1, 3)
    mol = RefMolecule(len(Z), Z.ctypes.data_as(POINTER(c_int)), pos.ctypes.data_as(POINTER(c_float)), 0)
    exp = RefExperiment()
    exp.wavelength = wavelength
    exp.bandwidth = bandwidth
    opts = RefOptions()
    opts.wavelength_samples = int(wavelength_samples)
    res = L.cuda_compute_pattern_on_list2(ctypes.byref(mol), _p(hkl), hkl.shape[0], float(B), ctypes.byref(exp),
                                          ctypes.byref(opts))
    n = hkl.shape[0]
    Fr = np.ctypeslib.as_array(ctypes.cast(res.contents.F, POINTER(c_float)), shape=(2 * n,)).copy()
    I = np.ctypeslib.as_array(res.contents.ints, shape=(n,)).copy()
    libc = ctypes.CDLL(None)
    for ptr in (res.contents.F, res.contents.ints, res.contents.HKL_list):
        libc.free(ctypes.cast(ptr, c_void_p))
    libc.free(ctypes.cast(res, c_void_p))
    return Fr[0::2] + 1j * Fr[1::2], I


# ---- spsim's own molecule.c / io.c (compiled into libspsim_ref.so)
def _ref_mol_setup():
    L = ref_lib()
    L.get_Molecule_from_pdb.restype = POINTER(RefMolecule)
    L.get_Molecule_from_pdb.argtypes = [ctypes.c_char_p]
    L.write_pdb_from_mol.argtypes = [ctypes.c_char_p, POINTER(RefMolecule)]
    L.origin_to_center_of_mass.argtypes = [POINTER(RefMolecule)]
    L.write_3D_array_to_vtk.argtypes = [c_void_p, c_int, c_int, c_int, ctypes.c_char_p]
    L.write_2D_array_to_vtk.argtypes = [c_void_p, c_int, c_int, ctypes.c_char_p]
    return L


def _mol_arrays(m):
    n = m.contents.natoms
    Z = np.ctypeslib.as_array(m.contents.atomic_number, shape=(max(n, 1),))[:n].copy()
    pos = np.ctypeslib.as_array(m.contents.pos, shape=(max(3 * n, 1),))[:3 * n].copy().reshape(-1, 3)
    return Z, pos


def ref_read_pdb(path):
    """spsim's get_Molecule_from_pdb (src/molecule.c:65-297): (Z int32 (N,), pos float32 (N,3))."""
    L = _ref_mol_setup()
    m = L.get_Molecule_from_pdb(path.encode())
    Z, pos = _mol_arrays(m)
    libc = ctypes.CDLL(None)
    libc.free(ctypes.cast(m.contents.atomic_number, c_void_p))
    libc.free(ctypes.cast(m.contents.pos, c_void_p))
    libc.free(ctypes.cast(m, c_void_p))
    return Z, pos


def _ref_molecule(Z, pos):
    Z = np.array(Z, np.int32)  # copies: the reference edits molecules in place
    pos = np.array(pos, np.float32).reshape(-1)
    return RefMolecule(len(Z), Z.ctypes.data_as(POINTER(c_int)), pos.ctypes.data_as(POINTER(c_float)), 0), Z, pos


def ref_write_pdb(path, Z, pos):
    """spsim's write_pdb_from_mol (src/molecule.c:359-379)."""
    L = _ref_mol_setup()
    m, Z, pos = _ref_molecule(Z, pos)
    L.write_pdb_from_mol(path.encode(), ctypes.byref(m))


def ref_center(Z, pos):
    """spsim's origin_to_center_of_mass (src/molecule.c:440-464) on a copy."""
    L = _ref_mol_setup()
    m, Z, p = _ref_molecule(Z, pos)
    L.origin_to_center_of_mass(ctypes.byref(m))
    return p.reshape(-1, 3).copy()


def ref_write_vtk(path, F, nx, ny, nz=None):
    """spsim's write_3D_array_to_vtk / write_2D_array_to_vtk (src/io.c)."""
    L = _ref_mol_setup()
    F = np.ascontiguousarray(F, np.float32)
    if nz is None:
        L.write_2D_array_to_vtk(_p(F), nx, ny, path.encode())
    else:
        L.write_3D_array_to_vtk(_p(F), nx, ny, nz, path.encode())


def hkl_3d_detector(nx, ny, nz, width, height, depth, distance, wavelength, center=(0.0, 0.0, 0.0)):
    """The oracle's 3-D detector grid (float32 (nx*ny*nz, 3))."""
    L = oracle_lib()
    out = np.zeros(3 * nx * ny * nz, np.float32)
    f = c_float
    L.oracle_hkl_3d_detector.argtypes = [c_int, c_int, c_int, f, f, f, f, f, f, f, f, c_void_p]
    L.oracle_hkl_3d_detector(nx, ny, nz, width, height, depth, distance, center[0], center[1], center[2], wavelength,
                             _p(out))
    return out.reshape(-1, 3)


def ref_hkl_3d_detector(nx, ny, nz, width, height, depth, distance, wavelength, center=(0.0, 0.0, 0.0)):
    """spsim's get_HKL_list_for_3d_detector (src/diffraction.c:325-369)."""
    L = _ref_setup()
    det = RefCCD(nx=nx, ny=ny, nz=nz, width=width, height=height, depth=depth, distance=distance,
                 center_x=center[0], center_y=center[1], center_z=center[2])
    exp = RefExperiment(wavelength=wavelength)
    n = c_int(0)
    L.get_HKL_list_for_3d_detector.restype = POINTER(c_float)
    L.get_HKL_list_for_3d_detector.argtypes = [POINTER(RefCCD), POINTER(RefExperiment), POINTER(c_int)]
    p = L.get_HKL_list_for_3d_detector(ctypes.byref(det), ctypes.byref(exp), ctypes.byref(n))
    out = np.ctypeslib.as_array(p, shape=(n.value * 3,)).copy().reshape(-1, 3)
    ctypes.CDLL(None).free(ctypes.cast(p, c_void_p))
    return out


def crystal(F, q, cell, size):
    """The oracle's FP64 crystal lattice sum: (F complex128, I float64)."""
    L = oracle_lib()
    q = np.ascontiguousarray(q, np.float64).reshape(-1, 3)
    Fr = np.ascontiguousarray(np.real(F), np.float64).copy()
    Fi = np.ascontiguousarray(np.imag(F), np.float64).copy()
    cell = np.ascontiguousarray(cell, np.float64).reshape(9)
    I = np.zeros(q.shape[0])
    L.oracle_crystal.argtypes = [ctypes.c_long, c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]
    L.oracle_crystal(q.shape[0], _p(q), _p(cell), int(size[0]), int(size[1]), int(size[2]), _p(Fr), _p(Fi), _p(I))
    return Fr + 1j * Fi, I


def ref_crystal(F, q, opts):
    """spsim's calculate_pattern_from_crystal (src/crystal.c:39-71), float, on copies."""
    L = ref_lib()
    n = q.shape[0]
    Fc = np.zeros(2 * n, np.float32)
    Fc[0::2], Fc[1::2] = np.real(F), np.imag(F)
    I = np.zeros(n, np.float32)
    qf = np.ascontiguousarray(q, np.float32).reshape(-1)
    L.calculate_pattern_from_crystal.argtypes = [c_void_p, c_void_p, c_void_p, c_int, POINTER(RefOptions)]
    L.calculate_pattern_from_crystal(_p(I), _p(Fc), _p(qf), n, ctypes.byref(opts))
    return Fc[0::2] + 1j * Fc[1::2], I


def ref_cell_matrix(opts):
    """spsim's crystal_cell_matrix (src/crystal.c:23-37)."""
    L = ref_lib()
    m = np.zeros(9, np.float32)
    L.crystal_cell_matrix.argtypes = [POINTER(RefOptions), c_void_p]
    L.crystal_cell_matrix(ctypes.byref(opts), _p(m))
    return m
