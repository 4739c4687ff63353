"""Crystal lattice (src/crystal.c): the cell matrix bit for bit against
spsim's own code, and the oracle's FP64 lattice sum against spsim's float
calculate_pattern_from_crystal.  Host code only: no GPU."""
import os

import numpy as np
import pytest

from conftest import intensity_errors
from oracle import oracle as O
from spsim_b200 import spsim as S

needs_ref = pytest.mark.skipif(not os.path.exists(O.REF_LIB), reason="oracle/_ref not built")

CELLS = [(1e-9, 1e-9, 1e-9, 90, 90, 90), (5.2e-9, 6.1e-9, 7.3e-9, 90, 90, 120),
         (3.1e-9, 4.7e-9, 5.9e-9, 81.5, 97.25, 103.75)]


def _ref_opts(cell, size=(1, 1, 1)):
    o = O.RefOptions()
    for k in range(6):
        o.crystal_cell[k] = cell[k]
    for k in range(3):
        o.crystal_size[k] = size[k]
    return o


@needs_ref
@pytest.mark.parametrize("cell", CELLS)
def test_cell_matrix_bit_exact(cell):
    want = O.ref_cell_matrix(_ref_opts(cell))
    opts = S.set_defaults()
    for k in range(6):
        opts.contents.crystal_cell[k] = cell[k]
    got = np.zeros(9, np.float32)
    S.crystal_cell_matrix(opts, got)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@needs_ref
@pytest.mark.parametrize("cell,size", [(CELLS[0], (2, 2, 2)), (CELLS[2], (3, 2, 4))])
def test_oracle_lattice_sum_against_reference(cell, size):
    rng = np.random.Generator(np.random.PCG64(8))
    q = rng.uniform(-6e8, 6e8, (3000, 3))
    F = (rng.normal(size=3000) + 1j * rng.normal(size=3000)).astype(np.complex64)
    cm = O.ref_cell_matrix(_ref_opts(cell))
    F64, I64 = O.crystal(F.astype(np.complex128), q.astype(np.float32).astype(np.float64), cm.astype(np.float64), size)
    Fr, Ir = O.ref_crystal(F, q, _ref_opts(cell, size))
    e_max, e_l2 = intensity_errors(Ir, I64)
    assert e_max < 1e-3 and e_l2 < 1e-5, (e_max, e_l2)  # the reference works in float
