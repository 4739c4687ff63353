"""The oracle's analytic FP64 vector-Jacobian product against FP64 central
differences of its own forward (h = 1e-4 Angstrom).  CPU only."""
import numpy as np
import pytest

from oracle import oracle as O
from spsim_b200 import synth


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


def test_oracle_vjp_matches_central_differences():
    Z, pos, occ, b, R, d, q, g = _case(n=12, nx=8, npat=1, bfac=True)
    pos64 = pos.astype(np.float64)
    dp, do, db = O.structure_factor_vjp(Z, pos64, q, g, occ=occ, bfac=b)
    h = 1e-14  # 1e-4 Angstrom

    def L(p, o=occ, bb=b):
        return float(np.dot(g, O.structure_factor(Z, p, q, occ=o, bfac=bb)[1]))

    for j in (0, 5, 11):
        for k in range(3):
            pp, pm = pos64.copy(), pos64.copy()
            pp[j, k] += h
            pm[j, k] -= h
            fd = (L(pp) - L(pm)) / (2 * h)
            assert fd == pytest.approx(dp[j, k], rel=1e-4, abs=1e-6 * np.abs(dp).max())
        o2, o3 = occ.astype(np.float64).copy(), occ.astype(np.float64).copy()
        o2[j] += 1e-6
        o3[j] -= 1e-6
        assert (L(pos64, o2) - L(pos64, o3)) / 2e-6 == pytest.approx(do[j], rel=1e-4, abs=1e-6 * np.abs(do).max())
        b2, b3 = b.astype(np.float64).copy(), b.astype(np.float64).copy()
        b2[j] += 1e-4
        b3[j] -= 1e-4
        assert (L(pos64, occ, b2) - L(pos64, occ, b3)) / 2e-4 == pytest.approx(db[j], rel=1e-4,
                                                                                 abs=1e-6 * np.abs(db).max())
