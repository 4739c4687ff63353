"""The structure-factor kernels' bounded waits give up instead of hanging.

Every atom tile reaches shared memory by a bulk copy that completes on an
mbarrier, and every wait on such a barrier has an iteration limit: on expiry
the kernel records an error word, waits (bounded) for its copies still in
flight and returns, and the host reports SPSIM_ERR_TIMEOUT.  The test hook
spsim_b200_debug_stall_first_copy makes each CTA arm its first barrier
without issuing the copy (a barrier that nothing completes) and shortens the
limit to ~10 ms.  Nothing faults and the context stays usable: with the hook
off again the next forward matches the FP64 oracle.
"""
import ctypes

import numpy as np
import pytest
import torch

from conftest import intensity_errors
from oracle import oracle as O
from spsim_b200 import _native, core, synth
from spsim_b200._native import SPSIM_ERR_TIMEOUT, SpsimError

pytestmark = pytest.mark.gpu

# one variant of each kernel form: compensated FP32 (0, 1), FP64 phase (2),
# FP64-anchored neighbour pairs (3) and quads (4)
FORMS = [(128, 4, 0), (128, 4, 1), (128, 4, 2), (128, 8, 3), (128, 8, 4)]
DET = dict(nx=64, ny=40, width=64 * 150e-6, height=40 * 150e-6, distance=0.1, wavelength=0.2e-9)


def _stall(on):
    _native.check(_native.lib().spsim_b200_debug_stall_first_copy(int(on)))


@pytest.mark.parametrize("variant", FORMS, ids=["form%d" % v[2] for v in FORMS])
def test_stalled_copy_reports_timeout_then_runs_normally(cuda, variant):
    Z, pos = synth.random_molecule(2000, 3e-9, 31)
    mol = core.Molecule(Z, pos)
    qs = core.QSet.from_detector(**DET)
    _, I64 = O.structure_factor(Z, pos.astype(np.float64), O.hkl_detector(**DET))
    side = torch.cuda.Stream()
    try:
        core.set_variant(*variant)
        _stall(True)
        try:
            # an asynchronous forward on the default stream (direct launches) and
            # one on a side stream (graph capture and replay): both report
            # through spsim_b200_synchronize
            for stream in (None, side):
                core.forward(mol, qs, precision="f32", stream=stream)
                with pytest.raises(SpsimError) as e:
                    core.synchronize(stream)
                assert e.value.status == SPSIM_ERR_TIMEOUT
            assert core.last_variant() == variant
        finally:
            _stall(False)
        for stream in (None, side):
            _, I = core.forward(mol, qs, precision="f32", stream=stream)
            core.synchronize(stream)
            e_max, e_l2 = intensity_errors(I.cpu().numpy(), I64)
            assert e_max < 1e-5 and e_l2 < 1e-6, (e_max, e_l2)
    finally:
        core.set_variant(-1)


def _host_sf(fn, Z, pos, hkl):
    n = hkl.shape[0]
    F = np.zeros(2 * n, np.float32)
    I = np.zeros(n, np.float32)
    p = ctypes.c_void_p
    Z = np.ascontiguousarray(Z, np.int32)
    pos = np.ascontiguousarray(pos, np.float32)
    hkl = np.ascontiguousarray(hkl, np.float32)
    st = fn(len(Z), Z.ctypes.data_as(p), pos.ctypes.data_as(p), None, None, 0.0, 0, None, n, hkl.ctypes.data_as(p),
            _native.PREC_F32, F.ctypes.data_as(p), I.ctypes.data_as(p))
    return st, I


def test_synchronous_host_calls_return_timeout(cuda):
    # the host-memory entry points wait for their work and return the status directly
    Z, pos = synth.random_molecule(1500, 2.5e-9, 33)
    hkl = O.hkl_detector(**DET).astype(np.float32)
    _, I64 = O.structure_factor(Z, pos.astype(np.float64), hkl.astype(np.float64))
    L = _native.lib()
    for fn in (L.spsim_b200_structure_factor_host, L.spsim_b200_structure_factor_host_noalloc):
        _stall(True)
        try:
            st, _ = _host_sf(fn, Z, pos, hkl)
        finally:
            _stall(False)
        assert st == SPSIM_ERR_TIMEOUT, st
        st, I = _host_sf(fn, Z, pos, hkl)
        assert st == 0
        e_max, e_l2 = intensity_errors(I, I64)
        assert e_max < 1e-5 and e_l2 < 1e-6, (e_max, e_l2)
