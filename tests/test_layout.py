"""The Python backend's structs have the reference layouts (include/config.h,
include/diffraction.h): same field names, offsets and sizes as the structs
the oracle uses to call spsim's own compiled code."""
import ctypes

import numpy as np

import pytest

from oracle import oracle as O
from spsim_b200 import spsim_pybackend as B

PAIRS = [(B.Molecule, O.RefMolecule), (B.Experiment, O.RefExperiment), (B.CCD, O.RefCCD),
         (B.Chem_Formula, O.RefChemFormula), (B.Options, O.RefOptions), (B.Diffraction_Pattern, O.RefPattern)]


@pytest.mark.parametrize("ours,ref", PAIRS)
def test_struct_layout_matches_reference(ours, ref):
    assert ctypes.sizeof(ours) == ctypes.sizeof(ref)
    assert [f for f, *_ in ours._fields_] == [f for f, *_ in ref._fields_]
    for (f, _t), _r in zip(ours._fields_, ref._fields_):
        assert getattr(ours, f).offset == getattr(ref, f).offset, f


def test_molecule_helpers_round_trip():
    from spsim_b200 import spsim

    Z = [6, 7, 8]
    pos = [[1e-10, 2e-10, 3e-10], [0.0, -1e-10, 5e-10], [4e-10, 4e-10, 4e-10]]
    mol = spsim.get_molecule_from_atoms(Z, pos)
    z2, p2 = spsim.get_atoms_from_molecule(mol)
    assert list(z2) == Z
    np.testing.assert_allclose(p2, np.array(pos), rtol=1e-6)
    B.free_mol(mol)


def test_loop_range_is_whole_range_in_one_process():
    assert B.get_my_loop_start_and_end(1234) == (0, 1234)
