"""Polychromatic patterns (spsim's spectrum kernel semantics,
src/diffraction.cu:415-476): the GPU path against the FP64 oracle, against
spsim's own CUDA spectrum kernel (compiled unchanged, its float error band),
and through the reference-shaped compute_sf / cuda_compute_pattern_on_list2
dispatch.  Tolerances are the structure-factor tests' own."""
import numpy as np
import pytest
import torch

from conftest import golden, intensity_errors
from oracle import oracle as O
from spsim_b200 import core, synth
from spsim_b200 import spsim as S

pytestmark = pytest.mark.gpu

TOL = {"fp64": (2e-7, 1e-7), "f32": (1e-5, 1e-6), "f32_fast": (2e-4, 1e-5)}


@pytest.mark.parametrize("precision", ["fp64", "f32", "f32_fast"])
@pytest.mark.parametrize("bw,S", [(0.1, 5), (0.4, 4), (0.02, 9)])
def test_spectrum_against_oracle(cuda, precision, bw, S):
    Z, pos = synth.random_molecule(3000, 3.2e-9, 5)
    d = dict(nx=64, ny=48, width=64 * 300e-6, height=48 * 300e-6, distance=0.1, wavelength=0.2e-9)
    q = O.hkl_detector(**d)
    mol = core.Molecule(Z, pos)
    qs = core.QSet.from_detector(**d)
    F, I = core.forward_spectrum(mol, qs, d["wavelength"], bw, S, precision=precision)
    torch.cuda.synchronize()
    F64, I64 = O.structure_factor_spectrum(Z, pos.astype(np.float64), q, d["wavelength"], bw, S)
    e_max, e_l2 = intensity_errors(I.cpu().numpy(), I64)
    assert e_max < TOL[precision][0] and e_l2 < TOL[precision][1], (e_max, e_l2)
    assert np.abs(F.cpu().numpy() - F64).max() < 10 * TOL[precision][0] * np.abs(F64).max()


def test_spectrum_with_rotation_b_factors_and_batch_graph(cuda):
    Z, pos = synth.random_molecule(1500, 2.5e-9, 6)
    rng = np.random.Generator(np.random.PCG64(6))
    b = rng.uniform(0, 30, len(Z)).astype(np.float32)
    d = dict(nx=40, ny=40, width=40 * 300e-6, height=40 * 300e-6, distance=0.1, wavelength=0.15e-9)
    R = synth.haar_rotations(1, 7)[0]
    q = O.hkl_detector(**d) @ R.T
    mol = core.Molecule(Z, pos, bfac=b)
    qs = core.QSet.from_detector(**d)
    F64, I64 = O.structure_factor_spectrum(Z, pos.astype(np.float64), q, d["wavelength"], 0.2, 5, bfac=b, B=10.0)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):  # captured once, then replayed from the graph
        for _ in range(2):
            F, I = core.forward_spectrum(mol, qs, d["wavelength"], 0.2, 5, rot=R, B=10.0, precision="f32")
    s.synchronize()
    core.synchronize(s)
    e_max, e_l2 = intensity_errors(I.cpu().numpy(), I64)
    assert e_max < 1e-5 and e_l2 < 1e-6, (e_max, e_l2)


def test_spectrum_against_reference_cuda_kernel(cuda):
    if O.ref_gpu_lib() is None:
        pytest.skip("oracle/_ref/libspsim_refgpu.so not built (make -C oracle refgpu)")
    g = golden("sf_small.npz")
    lam = float(g["det"][5])
    Fr, Ir = O.ref_gpu_pattern(g["Z"], g["pos"], g["hkl"], wavelength=lam, bandwidth=0.3, wavelength_samples=6)
    F64, I64 = O.structure_factor_spectrum(g["Z"], g["pos"].astype(np.float64), g["hkl"].astype(np.float64), lam,
                                           0.3, 6)
    F, I = core.forward_spectrum(core.Molecule(g["Z"], g["pos"]), core.QSet.from_list(g["hkl"]), lam, 0.3, 6)
    ref_err = intensity_errors(Ir, I64)  # the reference's float spectrum kernel against the FP64 restatement
    assert ref_err[0] < 1e-4 and ref_err[1] < 1e-5, ref_err
    r_max, r_l2 = intensity_errors(Ir, I.cpu().numpy().astype(np.float64))
    assert r_max < ref_err[0] + 2e-5 and r_l2 < ref_err[1] + 2e-6


def test_reference_dispatch_applies_the_spectrum(cuda):
    g = golden("sf_small.npz")
    lam = float(g["det"][5])
    n = g["hkl"].shape[0]
    mol = S.get_molecule_from_atoms(g["Z"], g["pos"])
    F64, I64 = O.structure_factor_spectrum(g["Z"], g["pos"].astype(np.float64), g["hkl"].astype(np.float64), lam,
                                           0.4, 5)
    _, Imono = O.structure_factor(g["Z"], g["pos"].astype(np.float64), g["hkl"].astype(np.float64))
    for use_cuda, want in ((1, I64), (2, Imono), (0, Imono)):
        opts = S.set_defaults()
        o = opts.contents
        o.verbosity_level = 0
        o.use_cuda = use_cuda
        o.wavelength_samples = 4
        o.experiment.contents.wavelength = lam
        o.experiment.contents.bandwidth = 0.4
        pat = S.compute_sf(mol, g["hkl"], n, opts)
        I = S.as_array(pat.contents.ints, n)
        e_max, _ = intensity_errors(I, want)
        assert e_max < 1e-5, (use_cuda, e_max)
        # the reference's CUDA path raises an even sample count by one in the options
        assert o.wavelength_samples == (5 if use_cuda == 1 else 4)
        S.free_diffraction_pattern(pat)
    S.free_mol(mol)
