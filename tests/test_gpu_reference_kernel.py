"""spsim's own CUDA path (src/diffraction.cu, cuda_compute_pattern_on_list2,
compiled unchanged for sm_100a by oracle/Makefile) as a GPU comparison point:
its accuracy against the FP64 oracle beside ours, and its speed beside ours on
the 50,000-atom / 1024^2 precision-stress workload.  Run with -s to see the
figures (one JSON line per measurement)."""
import json
import time

import numpy as np
import pytest
import torch

from conftest import golden, intensity_errors
from oracle import oracle as O
from spsim_b200 import core, synth

pytestmark = pytest.mark.gpu


def _need_ref_gpu():
    if O.ref_gpu_lib() is None:
        pytest.skip("oracle/_ref/libspsim_refgpu.so not built (make -C oracle refgpu)")


def test_reference_cuda_kernel_accuracy_beside_ours(cuda):
    _need_ref_gpu()
    g = golden("sf_small.npz")
    F64, I64 = O.structure_factor(g["Z"], g["pos"].astype(np.float64), g["hkl"].astype(np.float64))
    Fr, Ir = O.ref_gpu_pattern(g["Z"], g["pos"], g["hkl"])
    F, I = core.forward(core.Molecule(g["Z"], g["pos"]), core.QSet.from_list(g["hkl"]), precision="f32")
    ref_err = intensity_errors(Ir, I64)
    our_err = intensity_errors(I.cpu().numpy(), I64)
    print(json.dumps({"case": "sf_small", "reference_cuda": ref_err, "ours_f32": our_err}))
    # the reference kernel is float throughout: its own error band; ours is tighter
    assert ref_err[0] < 1e-3
    assert our_err[0] < 1e-5 and our_err[0] <= ref_err[0]


def test_reference_cuda_kernel_speed_and_error_on_precision_stress(cuda):
    _need_ref_gpu()
    w = synth.WORKLOADS["precision_50k"]
    Z, pos = synth.random_molecule(w["natoms"], w["radius"], w["seed"])
    d = w["det"]
    hkl = O.ref_hkl_detector(d["nx"], d["ny"], d["width"], d["height"], d["distance"], d["wavelength"])
    terms = float(len(Z)) * hkl.shape[0]
    # reference: one call, wall clock around it (its kernels are synchronous, 100 atoms per launch)
    torch.cuda.synchronize()
    t = time.perf_counter()
    Fr, Ir = O.ref_gpu_pattern(Z, pos, hkl)
    ref_s = time.perf_counter() - t
    # ours: the same float HKL list, device-resident, CUDA events around the forward
    mol = core.Molecule(Z, pos)
    qs = core.QSet.from_list(hkl)
    F = torch.empty(hkl.shape[0], dtype=torch.complex64, device="cuda")
    I = torch.empty(hkl.shape[0], device="cuda")
    core.forward(mol, qs, precision="f32", F=F, I=I)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(3):
        core.forward(mol, qs, precision="f32", F=F, I=I)
    b.record()
    torch.cuda.synchronize()
    our_s = a.elapsed_time(b) * 1e-3 / 3
    # ours through the host-buffer entry point (copies in and out, like the reference call)
    import ctypes

    from spsim_b200 import _native

    L = _native.lib()
    vp = ctypes.c_void_p
    Zi = np.ascontiguousarray(Z, np.int32)
    P = np.ascontiguousarray(pos, np.float32)
    Fh = np.empty(2 * hkl.shape[0], np.float32)
    Ih = np.empty(hkl.shape[0], np.float32)

    def host_call():
        st = L.spsim_b200_structure_factor_host(len(Zi), Zi.ctypes.data_as(vp), P.ctypes.data_as(vp), None, None,
                                                ctypes.c_float(0), 0, None, ctypes.c_int64(hkl.shape[0]),
                                                hkl.ctypes.data_as(vp), _native.PREC_F32, Fh.ctypes.data_as(vp),
                                                Ih.ctypes.data_as(vp))
        assert st == 0

    host_call()
    t = time.perf_counter()
    for _ in range(3):
        host_call()
    host_s = (time.perf_counter() - t) / 3
    # accuracy of both against FP64 on every 64th detector row
    rows = np.arange(0, d["ny"], 64)
    sel = (rows[:, None] * d["nx"] + np.arange(d["nx"])[None, :]).reshape(-1)
    _, I64 = O.structure_factor(Z, pos.astype(np.float64), hkl[sel].astype(np.float64))
    ref_err = intensity_errors(Ir[sel], I64)
    our_err = intensity_errors(I.cpu().numpy()[sel], I64)
    print(json.dumps({"case": "precision_50k", "terms": terms,
                      "reference_cuda": {"s": ref_s, "terms_per_s": terms / ref_s, "floored_max_rel": ref_err[0],
                                         "l2_rel": ref_err[1]},
                      "ours_f32": {"s": our_s, "terms_per_s": terms / our_s, "floored_max_rel": our_err[0],
                                   "l2_rel": our_err[1], "kernel": core.kernel_name()},
                      "ours_f32_host_buffers": {"s": host_s, "terms_per_s": terms / host_s},
                      "speedup_kernel": ref_s / our_s, "speedup_host_buffers": ref_s / host_s}))
    assert our_err[0] < 1e-5 and our_err[1] < 1e-6
    assert our_s < ref_s and host_s < ref_s
