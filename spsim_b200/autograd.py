"""torch.autograd wrapper: intensities I = |F|^2 as a differentiable function of
atom positions, occupancies and per-atom B factors.

    mol = Molecule(Z, pos0, occ=occ0, bfac=b0)        # element order and grid fixed here
    I = intensity(mol, qs, pos, occ, bfac, rots)       # (npat, npix) float32, CUDA
    loss = poisson_nll(I * scale, counts); loss.backward()

The forward writes the tensors into the molecule's device records and runs the
batched forward kernel; the backward runs the hand-written adjoint kernel,
which recomputes phases instead of storing atoms x pixels terms.  Gradients
come back in FP64 and are cast to the input dtypes.
"""
import torch

from . import core

__all__ = ["StructureFactorIntensity", "intensity", "poisson_nll", "l2_loss"]


class StructureFactorIntensity(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pos, occ, bfac, mol, qs, rots, precision, B):
        npat = 1 if rots is None else len(rots)
        mol.update_device(pos.detach(), occ.detach() if occ is not None else None,
                          bfac.detach() if bfac is not None else None)
        F, I = core.forward_batch([mol] * npat, [qs] * npat, rots=rots, B=B, precision=precision)
        Fc = torch.stack(F)
        ctx.mol, ctx.qs, ctx.rots, ctx.precision, ctx.B = mol, qs, rots, precision, B
        ctx.have_occ, ctx.have_b = occ is not None, bfac is not None
        ctx.dtypes = (pos.dtype, occ.dtype if occ is not None else None, bfac.dtype if bfac is not None else None)
        ctx.save_for_backward(Fc)
        return torch.stack(I)

    @staticmethod
    def backward(ctx, gI):
        (Fc,) = ctx.saved_tensors
        dpos, docc, dB = core.adjoint(ctx.mol, ctx.qs, Fc.reshape(-1), gI.reshape(-1).float(), rots=ctx.rots,
                                      B=ctx.B, precision=ctx.precision, want_occ=ctx.have_occ, want_b=ctx.have_b)
        return (dpos.to(ctx.dtypes[0]), docc.to(ctx.dtypes[1]) if ctx.have_occ else None,
                dB.to(ctx.dtypes[2]) if ctx.have_b else None, None, None, None, None, None)


def intensity(mol, qs, pos, occ=None, bfac=None, rots=None, precision="f32", B=0.0):
    """Differentiable (npat, npix) intensities; pos (N,3) metres, occ (N,), bfac (N,) A^2."""
    return StructureFactorIntensity.apply(pos, occ, bfac, mol, qs, rots, precision, B)


def poisson_nll(lam, counts, eps=0.0):
    """sum(lam - k log lam) (the Poisson negative log-likelihood up to a constant)."""
    return (lam - counts * torch.log(lam + eps)).sum()


def l2_loss(I, target):
    return ((I - target) ** 2).sum()
