"""The spsim command-line program on this library (spsim_b200/_lib/spsim,
src/spsim.c:374-415): spsim.conf in, spsim.confout, molout.pdb and the output
arrays out, as CXI files (read with the spec-based reader tests/h5read.py).
A PDB molecule with BIOMT operators checks the scattering factors the
program writes against the FP64 oracle."""
import os
import subprocess

import numpy as np
import pytest

import h5read
from conftest import GOLDEN, intensity_errors
from oracle import oracle as O
from spsim_b200 import spsim as S

pytestmark = pytest.mark.gpu

CLI = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "spsim_b200", "_lib", "spsim")

DETECTOR = """detector_distance = 1.000000e-01;
detector_width = 9.600000e-03;
detector_height = 7.200000e-03;
detector_pixel_width = 1.500000e-04;
detector_pixel_height = 1.500000e-04;
detector_quantum_efficiency = 1.500000e-01;
detector_electron_hole_production_energy = 5.800000e-19;
detector_readout_noise = 1.000000e+01;
detector_dark_current = 1.000000e-01;
detector_linear_full_well = 2.000000e+05;
detector_binning = 2;
detector_maximum_value = 65535.0;
experiment_wavelength = 2.00000e-10;
experiment_exposure_time = 1.000000e-13;
experiment_beam_intensity = 2.102500000e+30;
number_of_patterns = 2;
random_seed = 7;
output_scattering_factors = 1;
output_count = 1;
output_noiseless_count = 1;
output_solid_angles = 1;
"""


def _data(tmp_path, name):
    """The image of one CXI file (complex for the {r, i} compound)."""
    f = h5read.read(str(tmp_path / name))
    assert int(f["/cxi_version"]) == 150
    a = f["/entry_1/image_1/data"]
    return h5read.complex_of(a) if a.dtype.names else a


def _run(tmp_path, conf):
    (tmp_path / "spsim.conf").write_text(conf)
    r = subprocess.run([CLI], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    return r


def test_cli_formula_molecule(cuda, tmp_path):
    conf = 'number_of_dimensions = 2;\ninput_type = "chemical_formula";\n' \
           'chemical_formula = {\n  atom6 = 620;\n  atom7 = 170;\n  atom8 = 200;\n  atom16 = 10;\n};\n' \
           'box_type = "spherical";\nbox_dimension = 5.0e-09;\n' + DETECTOR
    _run(tmp_path, conf)
    # spsim.confout is the options as read, in the writer's format
    opts = S.set_defaults()
    S.read_options_file(str(tmp_path / "spsim.conf"), opts)
    S.write_options_file(str(tmp_path / "check.confout"), opts)
    assert (tmp_path / "spsim.confout").read_bytes() == (tmp_path / "check.confout").read_bytes()
    # molout.pdb carries the element in the atom-name columns 13-14 only (the
    # reference's writer format), so it is counted here, not read back
    atoms = [l for l in (tmp_path / "molout.pdb").read_text().splitlines() if l.startswith("ATOM")]
    names = [l[13:15] for l in atoms]
    assert len(atoms) == 1000 and [names.count(e) for e in ("C ", "N ", "O ", "S ")] == [620, 170, 200, 10]
    nx, ny = 64, 48
    for k in range(2):
        for name, shape, dtype in (("noiseless_photon_out", (ny, nx), np.float32), ("photon_out", (ny, nx), np.float32),
                                   ("scattering_factors", (ny, nx), np.complex64),
                                   ("solid_angles", (ny, nx), np.float32),
                                   ("counts_out", (ny // 2, nx // 2), np.float32),
                                   ("noiseless_counts_out", (ny // 2, nx // 2), np.float32)):
            a = _data(tmp_path, "%s-%05d.cxi" % (name, k))
            assert a.shape == shape and a.dtype == dtype and np.all(np.isfinite(a.view(np.float32)))
    p0 = _data(tmp_path, "photon_out-00000.cxi")
    p1 = _data(tmp_path, "photon_out-00001.cxi")
    assert not np.array_equal(p0, p1)  # independent noise per shot


@pytest.mark.parametrize("nfft", [0, 1], ids=["direct", "nfft"])
def test_cli_pdb_molecule_scattering_factors(cuda, tmp_path, nfft):
    rng = np.random.Generator(np.random.PCG64(11))
    lines = []
    ops = [np.eye(3), np.array([[0, -1, 0], [1, 0, 0], [0, 0, 1.0]])]
    for k, R in enumerate(ops):
        t = [0.0, 0.0, 0.0] if k == 0 else [12.0, -3.0, 5.0]
        for r in range(3):
            lines.append("REMARK 350   BIOMT%d %3d%10.6f%10.6f%10.6f     %10.5f\n" % (r + 1, k + 1, *R[r], t[r]))
    for i in range(800):
        e = ["C", "N", "O", "S"][rng.integers(4)]
        x, y, z = rng.uniform(-20, 20, 3)
        lines.append("ATOM  %5d  %-3s ALA A%4d    %8.3f%8.3f%8.3f  1.00 20.00          %2s\n"
                     % (i + 1, e, 1, x, y, z, e))
    (tmp_path / "mol.pdb").write_text("".join(lines) + "END\n")
    conf = 'number_of_dimensions = 2;\ninput_type = "pdb";\npdb_filename = "mol.pdb";\n' + DETECTOR
    if nfft:  # compute_sf's NFFT branch (src/spsim.c:119-123), through simulate_shot
        conf += "use_nfft_for_sf = 1;\n"
    _run(tmp_path, conf)
    m = S.get_Molecule_from_pdb(str(tmp_path / "mol.pdb"))
    n = m.contents.natoms
    Z = np.ctypeslib.as_array(m.contents.atomic_number, shape=(n,)).copy()
    pos = np.ctypeslib.as_array(m.contents.pos, shape=(3 * n,)).copy().reshape(-1, 3)
    S.free_mol(m)
    assert n == 1600
    q = O.hkl_detector(64, 48, 9.6e-3, 7.2e-3, 0.1, 2e-10)
    F64, I64 = O.structure_factor(Z, pos.astype(np.float64), q.astype(np.float32).astype(np.float64))
    F = _data(tmp_path, "scattering_factors-00000.cxi").reshape(-1)
    e_max, e_l2 = intensity_errors(np.abs(F.astype(np.complex128)) ** 2, I64)
    assert e_max < 1e-5 and e_l2 < 1e-6, (e_max, e_l2)
