"""Molecule files and VTK output (src/molecule.c, src/io.c, src/spsim.c:83-97):
ours against spsim's own code compiled unchanged into oracle/_ref (bit-exact
atoms and positions, byte-identical files).  Host code only: no GPU."""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O
from spsim_b200 import spsim as S

needs_ref = pytest.mark.skipif(not os.path.exists(O.REF_LIB), reason="oracle/_ref not built")


def _atom(serial, name, res, x, y, z, elem, het=False):
    rec = "HETATM" if het else "ATOM  "
    return "%s%5d %-4s %3s A%4d    %8.3f%8.3f%8.3f  1.00 20.00          %2s\n" % (rec, serial, name, res, 1, x, y, z,
                                                                                elem)


def _pdb(path, rng, n, biomt=None, extra_lines=()):
    elems = ["C", "N", "O", "S", "FE", "Zn", "CL", "H", "P", "Ca", "SE"]
    lines = ["HEADER    SYNTHETIC TEST MOLECULE\n", "REMARK   2 RESOLUTION. 2.00 ANGSTROMS.\n"]
    if biomt:
        for k, (R, t) in enumerate(biomt):
            for r in range(3):
                lines.append("REMARK 350   BIOMT%d %3d%10.6f%10.6f%10.6f     %10.5f\n"
                             % (r + 1, k + 1, R[r][0], R[r][1], R[r][2], t[r]))
    for i in range(n):
        e = elems[rng.integers(len(elems))]
        x, y, z = rng.uniform(-60, 60, 3)
        lines.append(_atom(i + 1, e[:2], "ALA", x, y, z, e.rjust(2), het=bool(rng.integers(5) == 0)))
        if i % 97 == 5:
            lines.append("TER\n")
    lines.extend(extra_lines)
    lines.append("END\n")
    with open(path, "w") as f:
        f.writelines(lines)


def _ours(path):
    m = S.get_Molecule_from_pdb(str(path))
    n = m.contents.natoms
    Z = np.ctypeslib.as_array(m.contents.atomic_number, shape=(max(n, 1),))[:n].copy()
    pos = np.ctypeslib.as_array(m.contents.pos, shape=(max(3 * n, 1),))[:3 * n].copy().reshape(-1, 3)
    S.free_mol(m)
    return Z, pos


def _rot(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


@needs_ref
def test_pdb_atoms_bit_exact(tmp_path):
    rng = np.random.Generator(np.random.PCG64(1))
    p = tmp_path / "a.pdb"
    _pdb(p, rng, 2500)  # more than the reader's initial 1024-atom arrays
    Zr, pr = O.ref_read_pdb(str(p))
    Z, pos = _ours(p)
    assert len(Z) == 2500
    np.testing.assert_array_equal(Z, Zr)
    assert np.array_equal(pos.view(np.uint32), pr.view(np.uint32))


@needs_ref
@pytest.mark.parametrize("first_identity", [True, False])
def test_pdb_biomt_expansion_bit_exact(tmp_path, first_identity):
    rng = np.random.Generator(np.random.PCG64(2))
    ops = [(np.eye(3), np.zeros(3))] if first_identity else []
    while len(ops) < 4:
        ops.append((_rot(rng), rng.uniform(-80, 80, 3)))
    p = tmp_path / "b.pdb"
    _pdb(p, rng, 300, biomt=ops)
    Zr, pr = O.ref_read_pdb(str(p))
    Z, pos = _ours(p)
    assert len(Z) == 4 * 300
    np.testing.assert_array_equal(Z, Zr)
    assert np.array_equal(pos.view(np.uint32), pr.view(np.uint32))


def test_unknown_element_is_skipped(tmp_path):
    p = tmp_path / "c.pdb"
    with open(p, "w") as f:
        f.write(_atom(1, "C1", "ALA", 1.0, 2.0, 3.0, " C"))
        f.write(_atom(2, "X1", "ALA", 4.0, 5.0, 6.0, "  "))  # blank element: skipped
        f.write(_atom(3, "N1", "ALA", 7.0, 8.0, 9.0, " N"))
        f.write("END\n")
    Z, pos = _ours(p)
    np.testing.assert_array_equal(Z, [6, 7])
    np.testing.assert_allclose(pos, np.float32([[1, 2, 3], [7, 8, 9]]) * np.float32(1e-10), rtol=1e-6)


@needs_ref
def test_write_pdb_byte_identical(tmp_path):
    rng = np.random.Generator(np.random.PCG64(3))
    Z = rng.choice([1, 6, 7, 8, 16, 26, 30, 79, 104], 700).astype(np.int32)
    pos = (rng.uniform(-9e-9, 9e-9, (700, 3))).astype(np.float32)
    O.ref_write_pdb(str(tmp_path / "ref.pdb"), Z, pos)
    mol = S.get_molecule_from_atoms(Z, pos)
    S.write_pdb_from_mol(str(tmp_path / "ours.pdb"), mol)
    S.free_mol(mol)
    assert (tmp_path / "ours.pdb").read_bytes() == (tmp_path / "ref.pdb").read_bytes()
    # and it reads back (2-character symbols, Angstrom with 3 decimals)
    Z2, pos2 = _ours(tmp_path / "ours.pdb")


@needs_ref
def test_center_of_mass_bit_exact():
    rng = np.random.Generator(np.random.PCG64(4))
    Z = rng.choice([6, 7, 8, 16], 5000).astype(np.int32)
    pos = rng.uniform(1e-9, 9e-9, (5000, 3)).astype(np.float32)
    want = O.ref_center(Z, pos)
    mol = S.get_molecule_from_atoms(Z, pos)
    S.origin_to_center_of_mass(mol)
    got = np.ctypeslib.as_array(mol.contents.pos, shape=(3 * 5000,)).copy().reshape(-1, 3)
    S.free_mol(mol)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@needs_ref
@pytest.mark.parametrize("shape", [(7, 5, None), (6, 4, 3)])
def test_vtk_byte_identical(tmp_path, shape):
    nx, ny, nz = shape
    n = nx * ny * (nz or 1)
    F = np.random.Generator(np.random.PCG64(5)).lognormal(0, 6, n).astype(np.float32)
    O.ref_write_vtk(str(tmp_path / "ref.vtk"), F, nx, ny, nz)
    if nz is None:
        S.write_2D_array_to_vtk(F, nx, ny, str(tmp_path / "ours.vtk"))
    else:
        S.write_3D_array_to_vtk(F, nx, ny, nz, str(tmp_path / "ours.vtk"))
    assert (tmp_path / "ours.vtk").read_bytes() == (tmp_path / "ref.vtk").read_bytes()


def test_molecule_from_formula_counts_and_box():
    form = S.Chem_Formula()
    zs = (ctypes.c_int * 3)(6, 7, 8)
    qs = (ctypes.c_int * 3)(500, 200, 300)
    form.n_elements, form.atomic_number, form.quantity = 3, zs, qs
    opts = S.set_defaults()
    o = opts.contents
    for box, d in ((1, 2e-8), (2, 1e-8)):
        o.box_type, o.box_dimension = box, d
        m = S.get_Molecule_from_formula(ctypes.byref(form), opts)
        n = m.contents.natoms
        Z = np.ctypeslib.as_array(m.contents.atomic_number, shape=(n,)).copy()
        pos = np.ctypeslib.as_array(m.contents.pos, shape=(3 * n,)).copy().reshape(-1, 3)
        S.free_mol(m)
        assert n == 1000 and list(np.bincount(Z)[[6, 7, 8]]) == [500, 200, 300]
        assert list(Z[:3]) == [6, 6, 6] and Z[-1] == 8  # formula order
        if box == 1:
            assert np.all(np.linalg.norm(pos.astype(np.float64), axis=1) <= d / 2 * (1 + 1e-6))
        else:
            assert pos.min() >= 0 and pos.max() < d
