"""Adjoint kernel and the autograd wrapper against the FP64 oracle's analytic
vector-Jacobian product, which is itself checked against FP64 central
differences (h = 1e-4 Angstrom)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from spsim_b200 import autograd, core, synth

pytestmark = pytest.mark.gpu


def _case(n=40, nx=20, npat=2, seed=3, bfac=False):
    Z, pos = synth.random_molecule(n, 1.2e-9, seed)
    rng = np.random.Generator(np.random.PCG64(seed))
    occ = rng.uniform(0.5, 1.0, n).astype(np.float32)
    b = rng.uniform(0.0, 30.0, n).astype(np.float32) if bfac else None
    R = synth.haar_rotations(npat, seed + 1)
    d = dict(nx=nx, ny=nx, width=nx * 600e-6, height=nx * 600e-6, distance=0.1, wavelength=0.2e-9)
    q0 = O.hkl_detector(**d)
    q = np.concatenate([q0 @ r.T for r in R])
    g = rng.normal(size=q.shape[0])
    return Z, pos, occ, b, R, d, q, g


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-6), ("f32", 1e-4), ("f32_fast", 1e-3)])
@pytest.mark.parametrize("bfac", [False, True])
def test_adjoint_kernel_matches_oracle_vjp(cuda, precision, tol, bfac):
    Z, pos, occ, b, R, d, q, g = _case(bfac=bfac)
    mol = core.Molecule(Z, pos, occ=occ, bfac=b)
    qs = core.QSet.from_detector(**d)
    F, I = core.forward_batch([mol] * len(R), [qs] * len(R), rots=R, precision=precision)
    Fc = torch.cat(F)
    G = torch.from_numpy(g.astype(np.float32)).cuda()
    dpos, docc, dB = core.adjoint(mol, qs, Fc, G, rots=R, precision=precision)
    torch.cuda.synchronize()
    dp, do, db = O.structure_factor_vjp(Z, pos.astype(np.float64), q, g.astype(np.float32).astype(np.float64),
                                        occ=occ, bfac=b)
    assert _rel(dpos.cpu().numpy(), dp) < tol
    assert _rel(docc.cpu().numpy(), do) < tol
    if bfac:
        assert _rel(dB.cpu().numpy(), db) < tol


@pytest.mark.parametrize("form", [1, 2])
def test_adjoint_forms_on_several_atom_blocks(cuda, form):
    # 1,500 atoms (several atom blocks per element, ragged last blocks) through
    # the compensated (form 1) and the FP64-phase (form 2) adjoint kernels
    Z, pos = synth.random_molecule(1500, 2.2e-9, 12)
    rng = np.random.Generator(np.random.PCG64(12))
    occ = rng.uniform(0.5, 1.0, len(Z)).astype(np.float32)
    b = rng.uniform(0.0, 30.0, len(Z)).astype(np.float32)
    R = synth.haar_rotations(2, 13)
    d = dict(nx=36, ny=30, width=36 * 300e-6, height=30 * 300e-6, distance=0.1, wavelength=0.2e-9)
    q0 = O.hkl_detector(**d)
    q = np.concatenate([q0 @ r.T for r in R])
    g = rng.normal(size=q.shape[0]).astype(np.float32)
    mol = core.Molecule(Z, pos, occ=occ, bfac=b)
    qs = core.QSet.from_detector(**d)
    try:
        core.set_variant(128, 4, form)
        F, I = core.forward_batch([mol] * len(R), [qs] * len(R), rots=R, precision="f32")
        dpos, docc, dB = core.adjoint(mol, qs, torch.cat(F), torch.from_numpy(g).cuda(), rots=R, precision="f32")
        torch.cuda.synchronize()
    finally:
        core.set_variant(-1)
    dp, do, db = O.structure_factor_vjp(Z, pos.astype(np.float64), q, g.astype(np.float64), occ=occ, bfac=b)
    assert _rel(dpos.cpu().numpy(), dp) < 1e-4
    assert _rel(docc.cpu().numpy(), do) < 1e-4
    assert _rel(dB.cpu().numpy(), db) < 1e-4


def test_autograd_poisson_refinement_gradient(cuda):
    Z, pos, occ, b, R, d, q, g = _case(n=60, nx=24, npat=3, seed=8, bfac=True)
    mol = core.Molecule(Z, pos, occ=occ, bfac=b)
    qs = core.QSet.from_detector(**d)
    p = torch.tensor(pos, dtype=torch.float64, device="cuda", requires_grad=True)
    o = torch.tensor(occ, device="cuda", requires_grad=True)
    bb = torch.tensor(b, device="cuda", requires_grad=True)
    I = autograd.intensity(mol, qs, p, o, bb, rots=R)
    scale = 100.0 / float(I.mean())
    rng = np.random.Generator(np.random.PCG64(2))
    counts = torch.from_numpy(rng.poisson(I.detach().cpu().numpy() * scale).astype(np.float32)).cuda()
    loss = autograd.poisson_nll(I * scale, counts, eps=1e-12)
    loss.backward()
    lam = I.detach().double().cpu().numpy().reshape(-1) * scale
    gI = scale * (1.0 - counts.double().cpu().numpy().reshape(-1) / (lam + 1e-12))
    dp, do, db = O.structure_factor_vjp(Z, pos.astype(np.float64), q, gI, occ=occ, bfac=b)
    assert _rel(p.grad.cpu().numpy(), dp) < 1e-4
    assert _rel(o.grad.double().cpu().numpy(), do) < 1e-4
    assert _rel(bb.grad.double().cpu().numpy(), db) < 1e-4


def test_refinement_positions_update_in_place(cuda):
    Z, pos, occ, b, R, d, q, g = _case(n=30, nx=16, npat=1)
    mol = core.Molecule(Z, pos)
    qs = core.QSet.from_detector(**d)
    shifted = pos.astype(np.float64) + 0.3e-10
    mol.update_device(torch.from_numpy(shifted).cuda())
    F, I = core.forward(mol, qs, rot=R[0])
    F64, I64 = O.structure_factor(Z, shifted, q)
    assert np.max(np.abs(I.cpu().numpy() - I64) / np.maximum(I64, 1e-3 * I64.mean())) < 1e-5


def test_adjoint_wide_phase_range_uses_fp64_rounding(cuda):
    # |q|max |r - c|max above 2^17 cycles: the FP64-phase adjoint leaves the
    # fixed-point phase word (and its amplitude/phase folding of the pixel
    # factor) for the FP64 rounding reduction
    rng = np.random.Generator(np.random.PCG64(21))
    Z = rng.choice([6, 7, 8], 48).astype(np.int32)
    pos = rng.uniform(-3e-5, 3e-5, (48, 3)).astype(np.float32)
    occ = rng.uniform(0.5, 1.0, 48).astype(np.float32)
    q = (rng.normal(size=(512, 3)) * 3e9).astype(np.float32)
    qr = np.linalg.norm(q.astype(np.float64), axis=1).max() * np.linalg.norm(pos - pos.mean(0), axis=1).max()
    assert qr > 2.0 ** 17
    g = rng.normal(size=512).astype(np.float32)
    mol = core.Molecule(Z, pos, occ=occ)
    qs = core.QSet.from_list(q)
    F, I = core.forward(mol, qs, precision="f32")
    dpos, docc, _ = core.adjoint(mol, qs, F, torch.from_numpy(g).cuda(), precision="f32")
    torch.cuda.synchronize()
    dp, do, _ = O.structure_factor_vjp(Z, pos.astype(np.float64), q.astype(np.float64), g.astype(np.float64), occ=occ)
    assert _rel(dpos.cpu().numpy(), dp) < 1e-4
    assert _rel(docc.cpu().numpy(), do) < 1e-4
