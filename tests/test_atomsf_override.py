"""spsim's ./atomsf.lib override (src/diffraction.c:118-177): a coefficient
file in the working directory replaces the compiled-in form-factor table for
every structure factor of the process.  Every row's a1 becomes -1, then each
record of the file replaces its element's row the first time the element
appears.  The file here is written by the test in the 5-line record layout
spsim reads (name; Z and, from column 24, c; a1..a4; b1..b4 in 16-column
fields; one more line), with carbon's coefficients altered, a second carbon
record that must be ignored, and iron left out (its a1 becomes -1).

Each library reads the file once per process, so every run is a subprocess
whose working directory holds the file.  CPU: spsim's own CPU path (compiled
from its sources) against the FP64 oracle with the same table.  GPU: the
library's forward and its allocation-free entry point against that oracle.
"""
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, intensity_errors
from oracle import oracle as O
from spsim_b200 import synth


def _table():
    base = O.atomsf_table()
    t = base.copy()
    t[6, 0] *= 1.3
    t[6, 5] *= 0.7
    t[6, 8] = 0.5
    return base, t


def _write_lib(path, t, decoy):
    with open(path, "w") as f:
        f.write("AD  synthetic coefficient file for the override test\n")
        f.write("AD  records: name / Z Z c / a1..a4 / b1..b4 / extra\n")
        for z, row in [(6, t[6]), (7, t[7]), (8, t[8]), (16, t[16]), (6, decoy)]:
            f.write("EL%d\n" % z)
            f.write("%5d%5d%13s%16.6f\n" % (z, z, "", row[8]))
            f.write("".join("%16.6f" % v for v in row[:4]) + "\n")
            f.write("".join("%16.6f" % v for v in row[4:8]) + "\n")
            f.write("%16.6f%16.6f\n" % (0.0, 0.0))


def _case(tmp_path):
    # compact, so that spsim's float phase stays accurate at |q| up to ~8e9 1/m
    Z, pos = synth.random_molecule(120, 0.8e-9, 88)
    Z = Z.copy()
    Z[::17] = 26  # iron: absent from the file
    hkl = (np.random.Generator(np.random.PCG64(88)).normal(size=(3000, 3)) * 2e9).astype(np.float32)
    base, t = _table()
    decoy = t[6] * 2.0
    _write_lib(tmp_path / "atomsf.lib", t, decoy)
    np.savez(tmp_path / "case.npz", Z=Z, pos=pos, hkl=hkl)
    return Z, pos, hkl, base


def _run(tmp_path, code):
    script = "import sys; sys.path.insert(0, %r)\nimport numpy as np\nd = np.load('case.npz')\n" % ROOT + code
    res = subprocess.run([sys.executable, "-c", script], cwd=str(tmp_path), capture_output=True, text=True,
                         timeout=600)
    assert res.returncode == 0, res.stderr[-3000:]
    return np.load(tmp_path / "out.npz")


def _oracle_with_file(tmp_path, Z, pos, hkl):
    t = O.atomsf_lib_table(str(tmp_path / "atomsf.lib"))
    try:
        O.set_atomsf_table(t)
        _, I64 = O.structure_factor(Z, pos.astype(np.float64), hkl.astype(np.float64))
    finally:
        O.reset_atomsf_table()
    return t, I64


def test_parser_follows_the_reference_rules(tmp_path):
    Z, pos, hkl, base = _case(tmp_path)
    t = O.atomsf_lib_table(str(tmp_path / "atomsf.lib"))
    _, want = _table()
    for z in (6, 7, 8, 16):
        np.testing.assert_array_equal(t[z], np.float32(["%.6f" % v for v in want[z]]).astype(np.float32))
    assert t[26, 0] == -1.0 and np.array_equal(t[26, 1:], base[26, 1:])
    assert np.all(t[:, 0][[z for z in range(100) if z not in (6, 7, 8, 16)]] == -1.0)


@pytest.mark.skipif(not O.ref_available(), reason="spsim's own sources are not built (oracle/_ref)")
def test_reference_cpu_path_reads_the_file_like_the_oracle(tmp_path):
    Z, pos, hkl, base = _case(tmp_path)
    # one atom at the origin per element: I = f_e(|q|)^2, which pins the table
    q1 = np.zeros((64, 3), np.float32)
    q1[:, 0] = np.linspace(0.0, 8e9, 64)
    out = _run(tmp_path, "from oracle import oracle as O\n"
                         "F, I = O.ref_pattern(d['Z'], d['pos'], d['hkl'])\n"
                         "q1 = np.zeros((64, 3), np.float32); q1[:, 0] = np.linspace(0.0, 8e9, 64)\n"
                         "f = [np.sqrt(O.ref_pattern(np.array([z], np.int32), np.zeros((1, 3), np.float32), q1)[1])"
                         " for z in (6, 7, 8, 16, 26)]\n"
                         "np.savez('out.npz', I=I, f=np.array(f))\n")
    t = O.atomsf_lib_table(str(tmp_path / "atomsf.lib"))
    f64 = np.array([[abs(O.scatt_factor(float(qq), z)) for qq in q1[:, 0]] for z in (6, 7, 8, 16, 26)])
    O.set_atomsf_table(t)
    try:
        f_file = np.array([[abs(O.scatt_factor(float(qq), z)) for qq in q1[:, 0]] for z in (6, 7, 8, 16, 26)])
    finally:
        O.reset_atomsf_table()
    err = np.abs(out["f"] - f_file).max(axis=1) / f_file.max(axis=1)
    assert np.all(err < 1e-6), err  # float evaluation of the same coefficients
    assert np.abs(f64 - f_file)[0].max() > 0.1  # carbon's row changed; the decoy record was ignored
    # the whole molecule, at spsim's own float error on this geometry
    _, I64 = _oracle_with_file(tmp_path, Z, pos, hkl)
    e_max, e_l2 = intensity_errors(out["I"], I64)
    assert e_max < 5e-5 and e_l2 < 2e-6, (e_max, e_l2)
    _, I_default = O.structure_factor(Z, pos.astype(np.float64), hkl.astype(np.float64))
    assert np.max(np.abs(I_default - I64) / np.maximum(I64, 1e-3 * I64.mean())) > 1e-2  # the file matters


@pytest.mark.gpu
def test_library_reads_the_file_like_the_reference(tmp_path):
    Z, pos, hkl, base = _case(tmp_path)
    out = _run(tmp_path, "import ctypes, torch\n"
                         "from spsim_b200 import core, _native\n"
                         "mol = core.Molecule(d['Z'], d['pos'])\n"
                         "qs = core.QSet.from_list(d['hkl'])\n"
                         "F, I = core.forward(mol, qs, precision='f32')\n"
                         "core.synchronize()\n"
                         "n = len(d['hkl']); I2 = np.zeros(n, np.float32); F2 = np.zeros(2 * n, np.float32)\n"
                         "Z = np.ascontiguousarray(d['Z'], np.int32); pos = np.ascontiguousarray(d['pos'])\n"
                         "hkl = np.ascontiguousarray(d['hkl']); p = ctypes.c_void_p\n"
                         "st = _native.lib().spsim_b200_structure_factor_host_noalloc(len(Z), Z.ctypes.data_as(p),"
                         " pos.ctypes.data_as(p), None, None, 0.0, 0, None, n, hkl.ctypes.data_as(p),"
                         " _native.PREC_F32, F2.ctypes.data_as(p), I2.ctypes.data_as(p))\n"
                         "assert st == 0, st\n"
                         "np.savez('out.npz', I=I.cpu().numpy(), I2=I2)\n")
    _, I64 = _oracle_with_file(tmp_path, Z, pos, hkl)
    for key in ("I", "I2"):
        e_max, e_l2 = intensity_errors(out[key], I64)
        assert e_max < 1e-5 and e_l2 < 1e-6, (key, e_max, e_l2)
