"""The allocation-free structure-factor entry point, called through the C ABI,
against the allocating one on the same inputs.

spsim_b200_structure_factor_host_noalloc serves callers that may not allocate
device memory while they run (their own fixed device-memory budget, or no
device-wide synchronising cudaMalloc / cudaFree per call): its scratch is a
static per-GPU array.  Two calls in a row with different molecules check that
nothing from the previous call leaks through the shared array.  Tolerances are
the structure-factor tests' own (tests/test_gpu_sf.py).  This file is collected
last so a failing run stops after every other test has run.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden, intensity_errors
from spsim_b200 import _native, synth

pytestmark = pytest.mark.gpu

TOL = {_native.PREC_F32: (1e-5, 1e-6), _native.PREC_F32_FAST: (2e-4, 1e-5), _native.PREC_FP64: (2e-7, 1e-7)}


def _call(fn, Z, pos, hkl, precision, B=0.0):
    n = hkl.shape[0]
    F = np.zeros(2 * n, np.float32)
    I = np.zeros(n, np.float32)
    Z = np.ascontiguousarray(Z, np.int32)
    pos = np.ascontiguousarray(pos, np.float32)
    hkl = np.ascontiguousarray(hkl, np.float32)
    p = ctypes.c_void_p
    st = fn(len(Z), Z.ctypes.data_as(p), pos.ctypes.data_as(p), None, None, ctypes.c_float(B), 0, None,
            ctypes.c_int64(n), hkl.ctypes.data_as(p), precision, F.ctypes.data_as(p), I.ctypes.data_as(p))
    return st, F[0::2] + 1j * F[1::2], I


def _fns():
    L = _native.lib()
    f = L.spsim_b200_structure_factor_host_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float,
                  ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_void_p]
    return L.spsim_b200_structure_factor_host, f


@pytest.mark.parametrize("precision", [_native.PREC_F32, _native.PREC_F32_FAST, _native.PREC_FP64])
def test_no_alloc_matches_allocating_entry_point_twice(cuda, precision):
    alloc, noalloc = _fns()
    g = golden("sf_small.npz")
    Z2, pos2 = synth.random_molecule(2500, 3e-9, 21)
    cases = [(g["Z"], g["pos"], g["hkl"], 20.0), (Z2, pos2, g["hkl"][:1500], 0.0)]
    for Z, pos, hkl, B in cases:  # two calls in a row through the shared scratch array
        s1, F1, I1 = _call(alloc, Z, pos, hkl, precision, B)
        s2, F2, I2 = _call(noalloc, Z, pos, hkl, precision, B)
        assert s1 == 0 and s2 == 0, (s1, s2)
        e_max, e_l2 = intensity_errors(I2, I1.astype(np.float64))
        assert e_max < TOL[precision][0] and e_l2 < TOL[precision][1], (e_max, e_l2)
        assert np.abs(F2 - F1).max() <= 10 * TOL[precision][0] * np.abs(F1).max()


def test_no_alloc_rejects_oversized_calls(cuda):
    _, noalloc = _fns()
    hkl = np.zeros((3_000_000, 3), np.float32)  # 3e6 pixels need more than the 64 MiB scratch
    st, _, _ = _call(noalloc, np.array([6], np.int32), np.zeros((1, 3), np.float32), hkl, _native.PREC_F32)
    assert st == _native.SPSIM_ERR_INVALID_ARG
