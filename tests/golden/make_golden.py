"""Generate the golden fixtures in tests/golden/ from spsim's own sources.

Runs only where the reference tree and oracle/_ref/libspsim_ref.so (built by
`make -C oracle ref REF=<spsim tree>`) are present; the fixtures are committed so that the
tests need neither.  Every array here is produced by spsim's own C code
(compiled unchanged against oracle/refstub), never by this project's code:

  sf_small.npz    HKL list of a 48x48 detector, scalar and SSE patterns of a
                  300-atom molecule, plus B-factor, delta-atom and Gaussian-beam
                  variants (src/diffraction.c:237-297, :770-968)
  sf_plain1k.npz  the 1000-atom / 256x256 workload, every 8th detector row
  chain.npz       Thomson (4 polarisations), solid angle (flat, spherical),
                  photons, electrons, binned real (no readout noise) and
                  noiseless outputs (src/diffraction.c:1109-1204, src/amplification.c)
  config/*.conf + *.confout   spsim.conf inputs and the reference's
                  write_options_file output after read_options_file
                  (src/config.c:89-642), with the parsed values as JSON

Usage: python tests/golden/make_golden.py
"""
import ctypes
import json
import os
import sys
import tempfile
from ctypes import POINTER, byref, c_float, c_int, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from spsim_b200 import synth  # noqa: E402


def sf_small():
    Z, pos = synth.random_molecule(300, 1.5e-9, 11)
    Z[5] = 0  # an atom the reference skips
    Z[17] = 26  # one iron atom: a fifth element
    kw = dict(nx=48, ny=48, width=48 * 200e-6, height=48 * 200e-6, distance=0.15, wavelength=0.25e-9)
    hkl = O.ref_hkl_detector(**kw)
    hkl_sph = O.ref_hkl_detector(spherical=True, **kw)
    F, I = O.ref_pattern(Z, pos, hkl)
    Fv, Iv = O.ref_pattern(Z, pos, hkl, vector=True)
    Fb, Ib = O.ref_pattern(Z, pos, hkl, B=20.0)
    Fd, Id = O.ref_pattern(Z, pos, hkl, delta_atoms=True)
    beam = (2.0e-9, 0.3e-9, -0.2e-9)
    Fg, Ig = O.ref_pattern(Z, pos, hkl, beam=beam)
    np.savez_compressed(os.path.join(HERE, "sf_small.npz"), Z=Z, pos=pos, hkl=hkl, hkl_spherical=hkl_sph,
                        det=np.array([kw["nx"], kw["ny"], kw["width"], kw["height"], kw["distance"],
                                      kw["wavelength"]]),
                        F=F.astype(np.complex64), I=I, F_vector=Fv.astype(np.complex64), I_vector=Iv,
                        F_B20=Fb.astype(np.complex64), I_B20=Ib, F_delta=Fd.astype(np.complex64), I_delta=Id,
                        beam=np.array(beam), F_beam=Fg.astype(np.complex64), I_beam=Ig)


def sf_plain1k():
    w = synth.WORKLOADS["plain_1k"]
    Z, pos = synth.random_molecule(w["natoms"], w["radius"], w["seed"])
    d = w["det"]
    hkl = O.ref_hkl_detector(d["nx"], d["ny"], d["width"], d["height"], d["distance"], d["wavelength"])
    rows = np.arange(0, d["ny"], 8)
    sel = (rows[:, None] * d["nx"] + np.arange(d["nx"])[None, :]).reshape(-1)
    F, I = O.ref_pattern(Z, pos, hkl[sel])
    np.savez_compressed(os.path.join(HERE, "sf_plain1k.npz"), Z=Z, pos=pos, rows=rows, hkl=hkl[sel],
                        F=F.astype(np.complex64), I=I)


def _arr(p, n):
    return np.ctypeslib.as_array(p, shape=(n,)).copy()


def chain():
    L = O._ref_setup()
    L.calculate_thomson_correction.argtypes = [POINTER(O.RefCCD), POINTER(O.RefExperiment)]
    L.calculate_pixel_solid_angle.argtypes = [POINTER(O.RefCCD)]
    L.calculate_photons_per_pixel.argtypes = [POINTER(O.RefPattern), POINTER(O.RefOptions)]
    L.calculate_electrons_per_pixel.argtypes = [POINTER(O.RefCCD), POINTER(O.RefExperiment)]
    L.calculate_real_detector_output.argtypes = [POINTER(O.RefCCD), POINTER(O.RefExperiment)]
    L.calculate_noiseless_detector_output.argtypes = [POINTER(O.RefCCD), POINTER(O.RefExperiment)]
    nx, ny = 40, 36
    base = dict(nx=nx, ny=ny, nz=1, width=nx * 110e-6, height=ny * 110e-6, distance=0.05, pixel_width=110e-6,
                pixel_height=110e-6, center_x=0.4e-3, center_y=-0.3e-3, quantum_efficiency=0.8,
                electron_hole_production_energy=5.8e-19, readout_noise=0.0, dark_current=30.0,
                linear_full_well=2e5, maximum_value=65535.0, binning_x=2, binning_y=3, binning_z=1)
    out = {}
    for pol in range(4):
        det = O.RefCCD(**base)
        exp = O.RefExperiment(wavelength=0.2e-9, polarization=pol, beam_intensity=1e30, exposure_time=1e-3)
        L.calculate_thomson_correction(byref(det), byref(exp))
        out["thomson_%d" % pol] = _arr(det.thomson_correction, nx * ny)
    for sph in (0, 1):
        det = O.RefCCD(spherical=sph, **base)
        L.calculate_pixel_solid_angle(byref(det))
        out["solid_angle_%d" % sph] = _arr(det.solid_angle, nx * ny)
    # photons from a given intensity pattern, with the polarised Thomson factor
    rng = np.random.Generator(np.random.PCG64(5))
    ints = (rng.exponential(size=nx * ny) * 1e4).astype(np.float32)
    det = O.RefCCD(**base)
    exp = O.RefExperiment(wavelength=0.2e-9, polarization=3, beam_intensity=2.1e30, exposure_time=1e-3)
    opts = O.RefOptions()
    opts.detector = ctypes.pointer(det)
    opts.experiment = ctypes.pointer(exp)
    pat = O.RefPattern()
    pat.ints = ints.ctypes.data_as(POINTER(c_float))
    L.calculate_photons_per_pixel(byref(pat), byref(opts))
    out["ints"] = ints
    out["photons"] = _arr(det.photons_per_pixel, nx * ny)
    counts = rng.poisson(np.maximum(out["photons"], 0) * 0.8).astype(np.float32)
    det.photon_count = counts.ctypes.data_as(POINTER(c_float))
    L.calculate_electrons_per_pixel(byref(det), byref(exp))
    out["counts"] = counts
    out["electrons"] = _arr(det.electrons_per_pixel, nx * ny)
    L.calculate_real_detector_output(byref(det), byref(exp))
    L.calculate_noiseless_detector_output(byref(det), byref(exp))
    nb = (nx // 2) * (ny // 3)
    out["real_output"] = _arr(det.real_output, nb)
    out["noiseless_output"] = _arr(det.noiseless_output, nb)
    out["params"] = np.array([nx, ny, base["width"], base["height"], base["distance"], base["pixel_width"],
                              base["pixel_height"], base["center_x"], base["center_y"], 0.8, 5.8e-19, 30.0, 2e5,
                              65535.0, 2, 3, 0.2e-9, 2.1e30, 1e-3])
    np.savez_compressed(os.path.join(HERE, "chain.npz"), **out)


CONFS = {
    "example": """# the example of spsim's own tree, without its missing PDB file
number_of_dimensions = 2;
input_type = "chemical_formula";
chemical_formula = {
  atom6 = 620;
  atom7 = 170;
  atom8 = 200;
  atom16 = 10;
};
detector_distance = 1.000000e-02;
detector_width = 2.680000e-02;
detector_height = 2.600000e-02;
detector_pixel_width = 4.000000e-05;
detector_pixel_height = 4.000000e-05;
detector_quantum_efficiency = 1.500000e-01;
detector_electron_hole_production_energy = 5.800000e-19;
detector_readout_noise = 1.000000e+01;
detector_dark_current = 1.000000e-01;
detector_linear_full_well = 2.000000e+05;
detector_binning = 1;
detector_maximum_value = 65535.0;
experiment_wavelength = 1.00000e-10;
experiment_exposure_time = 1.000000e-13;
#1e20 photons, 100um^2
experiment_beam_intensity = 2.102500000e+30;
crystal_size_a = 2;
crystal_size_b = 2;
crystal_size_c = 2;
crystal_cell_a = 1.0E-9;
crystal_cell_b = 1.0E-9;
crystal_cell_c = 1.0E-9;
""",
    "quirks": """/* integer literal for a float key reads as 0 (doc/UserManual.tex:91-93) */
input_type = "pdb";
pdb_filename = "mol \\"a\\".pdb";
detector_distance = 1;
detector_width : 0.0192;   // colon form
detector_height = 0.0192;
detector_pixel_width = 75.0e-6;
detector_pixel_height = 75.0E-6;
detector_binning_x = 2;
detector_binning_y = 4;
experiment_photon_energy = 8000.0;
experiment_polarization = "unpolarized";
experiment_focal_diameter = 1.0e-6;
experiment_beam_energy = 1.0e-3;
phi = 0.5; theta = 1.2; psi = -0.3;
random_orientation = 0;
number_of_patterns = 3;
b_factor = 15.5;
use_cuda = 0;
random_seed = 42;
verbosity_level = 0;
output_count = 1;
list_key = (1, 2.0, "x");
array_key = [1, 2, 3];
flag = true;
""",
}

OPTION_FIELDS = ["input_type", "pdb_filename", "box_type", "box_dimension", "b_factor", "euler_orientation",
                 "random_orientation", "n_patterns", "vectorize", "delta_atoms", "use_cuda", "wavelength_samples",
                 "random_seed", "output_photons", "output_count", "verbosity_level", "crystal_size", "crystal_cell"]
DET_FIELDS = ["distance", "width", "height", "depth", "pixel_width", "pixel_height", "quantum_efficiency",
              "electron_hole_production_energy", "readout_noise", "dark_current", "linear_full_well", "binning_x",
              "binning_y", "binning_z", "nx", "ny", "nz", "maximum_value", "spherical"]
EXP_FIELDS = ["wavelength", "exposure_time", "beam_intensity", "photon_energy", "focal_diameter", "beam_energy",
              "polarization"]


def _val(v):
    if isinstance(v, bytes):
        return v.decode()
    if hasattr(v, "__len__") and not isinstance(v, str):
        return [float(x) for x in v]
    return float(v) if isinstance(v, float) else v


def options_dict(o):
    d = {k: _val(getattr(o, k)) for k in OPTION_FIELDS}
    d.update({"detector." + k: _val(getattr(o.detector.contents, k)) for k in DET_FIELDS})
    d.update({"experiment." + k: _val(getattr(o.experiment.contents, k)) for k in EXP_FIELDS})
    cf = o.chem_formula.contents
    d["chem_formula"] = [[cf.atomic_number[i], cf.quantity[i]] for i in range(cf.n_elements)]
    return d


def config():
    L = O._ref_setup()
    L.read_options_file.argtypes = [ctypes.c_char_p, POINTER(O.RefOptions)]
    L.write_options_file.argtypes = [ctypes.c_char_p, POINTER(O.RefOptions)]
    cdir = os.path.join(HERE, "config")
    os.makedirs(cdir, exist_ok=True)
    parsed = {}
    with tempfile.TemporaryDirectory() as td:
        for name, text in CONFS.items():
            src = os.path.join(cdir, name + ".conf")
            with open(src, "w") as f:
                f.write(text)
            o = L.set_defaults()
            L.read_options_file(src.encode(), o)
            dst = os.path.join(td, name + ".confout")
            L.write_options_file(dst.encode(), o)
            with open(dst) as f, open(os.path.join(cdir, name + ".confout"), "w") as g:
                g.write(f.read())
            parsed[name] = options_dict(o.contents)
        o = L.set_defaults()
        dst = os.path.join(td, "defaults.confout")
        L.write_options_file(dst.encode(), o)
        with open(dst) as f, open(os.path.join(cdir, "defaults.confout"), "w") as g:
            g.write(f.read())
        parsed["defaults"] = options_dict(o.contents)
    with open(os.path.join(cdir, "parsed.json"), "w") as f:
        json.dump(parsed, f, indent=1, sort_keys=True)


def atomsf_table():
    """The reference's compiled-in coefficient table, read from its own source."""
    ref = os.environ.get("SPSIM_REFERENCE")
    if not ref:
        sys.exit("set SPSIM_REFERENCE to the spsim source tree")
    import re
    text = open(os.path.join(ref, "include", "atomsf.cdata")).read()
    rows = [[float(v) for v in r.split(",")] for r in re.findall(r"\{([^{}]*)\}", text)]
    np.save(os.path.join(HERE, "atomsf_reference.npy"), np.array(rows, np.float32))


if __name__ == "__main__":
    if not O.ref_available():
        sys.exit("build the reference first: make -C oracle ref REF=<spsim tree>")
    sf_small()
    sf_plain1k()
    chain()
    config()
    atomsf_table()
    print("golden fixtures written to", HERE)
