"""The oracle's 3-D (volume) detector grid against spsim's own
get_HKL_list_for_3d_detector (src/diffraction.c:325-369), bit for bit."""
import os

import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.skipif(not os.path.exists(O.REF_LIB), reason="oracle/_ref not built")
@pytest.mark.parametrize("shape,center", [((8, 6, 5), (1e-4, -2e-4, 3e-4)), ((16, 16, 16), (0.0, 0.0, 0.0)),
                                          ((1, 7, 3), (0.0, 5e-5, 0.0))])
def test_volume_grid_bit_exact(shape, center):
    nx, ny, nz = shape
    args = (nx, ny, nz, 1e-2, 8e-3, 6e-3, 0.12, 1.5e-10)
    a = O.hkl_3d_detector(*args, center=center)
    b = O.ref_hkl_3d_detector(*args, center=center)
    assert a.shape == (nx * ny * nz, 3)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
