"""The crystal lattice sum on the GPU (calculate_pattern_from_crystal,
src/crystal.c:39-71) against the FP64 oracle and against spsim's own float
version."""
import numpy as np
import pytest

from conftest import golden, intensity_errors
from oracle import oracle as O
from spsim_b200 import spsim as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cell,size", [((1e-9, 1e-9, 1e-9, 90, 90, 90), (2, 2, 2)),
                                       ((3.1e-9, 4.7e-9, 5.9e-9, 81.5, 97.25, 103.75), (5, 3, 4))])
def test_lattice_sum_against_oracle_and_reference(cuda, cell, size):
    g = golden("sf_small.npz")
    q = g["hkl"].astype(np.float32)
    F = g["F"].astype(np.complex64)  # the reference's own float pattern as input
    opts = S.set_defaults()
    o = opts.contents
    o.verbosity_level = 0
    for k in range(6):
        o.crystal_cell[k] = cell[k]
    for k in range(3):
        o.crystal_size[k] = size[k]
    cm = np.zeros(9, np.float32)
    S.crystal_cell_matrix(opts, cm)
    n = q.shape[0]
    Fbuf = np.zeros(2 * n, np.float32)
    Fbuf[0::2], Fbuf[1::2] = F.real, F.imag
    I = np.zeros(n, np.float32)
    S.calculate_pattern_from_crystal(I.ctypes.data_as(S.POINTER(S.c_float)),
                                     Fbuf.ctypes.data_as(S.POINTER(S.Complex)), q, n, opts)
    F64, I64 = O.crystal(F.astype(np.complex128), q.astype(np.float64), cm.astype(np.float64), size)
    e_max, e_l2 = intensity_errors(I, I64)
    assert e_max < 1e-5 and e_l2 < 1e-6, (e_max, e_l2)
    Fo = Fbuf[0::2] + 1j * Fbuf[1::2]
    assert np.abs(Fo - F64).max() < 1e-5 * np.abs(F64).max()
    ro = O.RefOptions()
    for k in range(6):
        ro.crystal_cell[k] = cell[k]
    for k in range(3):
        ro.crystal_size[k] = size[k]
    _, Ir = O.ref_crystal(F, q, ro)
    r_max, _ = intensity_errors(Ir, I64)
    assert intensity_errors(I, Ir)[0] < r_max + 1e-5
