"""Drop-in for spsim's Python module (src/spsim.py): the backend's names plus
the convenience helpers, with numpy in place of libspimage images."""
import numpy as np

from .spsim_pybackend import *  # noqa: F401,F403 - the module re-exports the backend, as spsim.py does
from .spsim_pybackend import add_atom_to_mol, alloc_mol

__version__ = "0.1.0"


def get_molecule_from_atoms(atomic_numbers=None, atomic_positions=None):
    """A Molecule (ctypes pointer) from atomic numbers and (N,3) positions in metres (src/spsim.py:23-27)."""
    mol = alloc_mol()
    for j, (x, y, z) in zip(atomic_numbers, atomic_positions):
        add_atom_to_mol(mol, int(j), float(x), float(y), float(z))
    return mol


def get_atoms_from_molecule(mol):
    """(atomic numbers int32 (N,), positions float64 (N,3)) of a Molecule (src/spsim.py:29-42)."""
    m = mol.contents
    anum = np.ctypeslib.as_array(m.atomic_number, shape=(m.natoms,)).astype(np.int32, copy=True)
    pos = np.ctypeslib.as_array(m.pos, shape=(m.natoms * 3,)).astype(np.float64).reshape(m.natoms, 3)
    return anum, pos
