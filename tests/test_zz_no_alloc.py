"""The allocation-free structure-factor entry point, called through the C ABI,
against the allocating one and against the FP64 oracle on the same inputs.

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
from oracle import oracle as O
from spsim_b200 import _native, synth

pytestmark = pytest.mark.gpu

TOL = {_native.PREC_F32: (1e-5, 1e-6), _native.PREC_F32_FAST: (2e-4, 1e-5), _native.PREC_FP64: (2e-7, 1e-7)}


def _arr(a, dtype):
    return None if a is None else np.ascontiguousarray(a, dtype)


def _call(fn, Z, pos, hkl, precision, B=0.0, occ=None, bfac=None, beam=None, delta_atoms=0):
    n = hkl.shape[0]
    F = np.zeros(2 * n, np.float32)
    I = np.zeros(n, np.float32)
    Z, pos, hkl = _arr(Z, np.int32), _arr(pos, np.float32), _arr(hkl, np.float32)
    occ, bfac, beam = _arr(occ, np.float32), _arr(bfac, np.float32), _arr(beam, np.float32)
    p = ctypes.c_void_p

    def ptr(a):
        return a.ctypes.data_as(p) if a is not None else None

    st = fn(len(Z), ptr(Z), ptr(pos), ptr(occ), ptr(bfac), B, int(delta_atoms), ptr(beam), n, ptr(hkl), precision,
            ptr(F), ptr(I))
    return st, F[0::2] + 1j * F[1::2], I


def _fns():
    L = _native.lib()
    return L.spsim_b200_structure_factor_host, L.spsim_b200_structure_factor_host_noalloc


def _check(Z, pos, hkl, precision, **kw):
    alloc, noalloc = _fns()
    s1, F1, I1 = _call(alloc, Z, pos, hkl, precision, **kw)
    s2, F2, I2 = _call(noalloc, Z, pos, hkl, precision, **kw)
    assert s1 == 0 and s2 == 0, (s1, s2, _native.lib().spsim_b200_last_error())
    # against the allocating entry point
    e_max, e_l2 = intensity_errors(I2, I1.astype(np.float64))
    assert e_max < TOL[precision][0] and e_l2 < TOL[precision][1], ("vs allocating", e_max, e_l2)
    assert np.abs(F2 - F1).max() <= 10 * TOL[precision][0] * np.abs(F1).max()
    # against the FP64 oracle
    okw = dict(B=kw.get("B", 0.0), occ=kw.get("occ"), bfac=kw.get("bfac"), beam=kw.get("beam"),
               delta_atoms=bool(kw.get("delta_atoms", 0)))
    F64, I64 = O.structure_factor(Z, np.asarray(pos, np.float32).astype(np.float64), hkl.astype(np.float64), **okw)
    e_max, e_l2 = intensity_errors(I2, I64)
    assert e_max < TOL[precision][0] and e_l2 < TOL[precision][1], ("vs oracle", e_max, e_l2)


@pytest.mark.parametrize("precision", [_native.PREC_F32, _native.PREC_F32_FAST, _native.PREC_FP64])
def test_no_alloc_matches_allocating_entry_point_and_oracle_twice(cuda, precision):
    g = golden("sf_small.npz")
    Z2, pos2 = synth.random_molecule(2500, 3e-9, 21)
    d = dict(nx=64, ny=40, width=64 * 150e-6, height=40 * 150e-6, distance=0.1, wavelength=0.2e-9)
    det = O.hkl_detector(**d).astype(np.float32)  # neighbour pairs: the pair form where FP32 admits it
    # two calls in a row through the shared scratch array
    _check(g["Z"], g["pos"], g["hkl"], precision, B=20.0)
    _check(Z2, pos2, det, precision)


@pytest.mark.parametrize("precision", [_native.PREC_F32, _native.PREC_FP64])
def test_no_alloc_weights_b_factors_beam_and_delta_atoms(cuda, precision):
    # occupancies, per-atom B factors and a Gaussian beam (the atom weights
    # occ sqrt(illumination) and the per-atom B kernels), then delta atoms
    g = golden("sf_plain1k.npz")
    rng = np.random.Generator(np.random.PCG64(23))
    n = len(g["Z"])
    occ = rng.uniform(0.3, 1.0, n).astype(np.float32)
    bfac = rng.uniform(0.0, 40.0, n).astype(np.float32)
    beam = np.array([3e-9, 0.4e-9, -0.3e-9], np.float32)
    _check(g["Z"], g["pos"], g["hkl"], precision, occ=occ, bfac=bfac, beam=beam)
    _check(g["Z"], g["pos"], g["hkl"], precision, delta_atoms=1)


def test_no_alloc_wide_phase_range(cuda):
    # |q|max |r - c|max above 2^17 cycles: the FP64-phase form reduces by FP64
    # rounding, as the allocating call does (no SPSIM_ERR_RANGE below 2^48)
    rng = np.random.Generator(np.random.PCG64(5))
    Z = rng.choice([6, 7, 8, 16], 64).astype(np.int32)
    pos = rng.uniform(-3e-5, 3e-5, (64, 3)).astype(np.float32)
    hkl = (rng.normal(size=(2048, 3)) * 3e9).astype(np.float32)
    qr = np.linalg.norm(hkl.astype(np.float64), axis=1).max() * np.linalg.norm(pos - pos.mean(0), axis=1).max()
    assert qr > 2.0 ** 17
    _check(Z, pos, hkl, _native.PREC_F32)


def test_no_alloc_rejects_oversized_calls(cuda):
    _, noalloc = _fns()
    L = _native.lib()
    # 3e6 pixels, then 1e6 atoms: each needs more than the 64 MiB scratch
    hkl = np.zeros((3_000_000, 3), np.float32)
    st, _, _ = _call(noalloc, np.array([6], np.int32), np.zeros((1, 3), np.float32), hkl, _native.PREC_F32)
    assert st == _native.SPSIM_ERR_INVALID_ARG
    assert b"device scratch" in L.spsim_b200_last_error()
    Z = np.full(1_000_000, 6, np.int32)
    pos = np.random.default_rng(2).normal(size=(1_000_000, 3)).astype(np.float32) * 1e-8
    st, _, _ = _call(noalloc, Z, pos, hkl[:16], _native.PREC_F32)
    assert st == _native.SPSIM_ERR_INVALID_ARG
    assert b"1000000 atoms" in L.spsim_b200_last_error()
    # a call within the limit still works afterwards
    g = golden("sf_small.npz")
    _check(g["Z"], g["pos"], g["hkl"], _native.PREC_F32)
