"""The NUFFT structure factor's algorithm and parameter rule on the CPU: a
small numpy restatement of its four steps (spread, deconvolve and pad, FFT,
interpolate and deconvolve) with the library's choices (upsampling 1.5 for
the spreading grid and 2 for the FFT grid, exponential-of-semicircle kernels,
interpolation width w2 = ceil(-log10 eps) + 1 and spreading width w2 + 3)
meets the requested relative error against the FP64 direct sum of the
oracle within a factor of 4 (measured 1.3x at 1e-6, 2.4x at 1e-8 here).
Test infrastructure only: the library's kernels are checked on the GPU by
tests/test_gpu_nufft.py."""
import numpy as np
import pytest

from oracle import oracle as O


def _es(u, w, beta):
    t = 2.0 * u / w
    a = 1.0 - t * t
    return np.where(a >= 0, np.exp(beta * (np.sqrt(np.clip(a, 0, None)) - 1.0)), 0.0)


def _es_hat(xi, w, beta, d=0.01):
    u = np.arange(int(np.floor(0.5 * w / d)) + 1) * d
    c = _es(u, w, beta) * d * np.where(np.arange(len(u)) == 0, 1.0, 2.0)
    return np.cos(2 * np.pi * np.outer(np.atleast_1d(xi), u)) @ c


def _nufft(x, c, q, eps):
    w2 = int(np.ceil(-np.log10(eps))) + 1
    w1 = w2 + 3
    s1, s2 = 1.5, 2.0
    b1, b2 = 0.97 * np.pi * w1 * (1 - 0.5 / s1), 0.97 * np.pi * w2 * (1 - 0.5 / s2)
    X = np.abs(x).max() * 1.05 + 1e-30
    lo, hi = q.min(0), q.max(0)
    cq, S = 0.5 * (lo + hi), np.maximum(0.5 * (hi - lo), 1e-3 / X)
    h = 1.0 / (2 * s1 * S)
    n1 = np.ceil(2 * X / h).astype(int) + w1 + 2
    n1 += n1 % 2
    n2 = np.ceil(s2 * n1).astype(int)
    n2 += n2 % 2
    cp = c * np.exp(-2j * np.pi * (x @ cq))
    # 1. spread
    grid = np.zeros(tuple(n1[::-1]), complex)
    s = x / h + n1 / 2
    l0 = np.ceil(s - w1 / 2).astype(int)
    for j in range(len(x)):
        k = [_es(s[j, d] - (l0[j, d] + np.arange(w1)), w1, b1) for d in range(3)]
        grid[l0[j, 2]:l0[j, 2] + w1, l0[j, 1]:l0[j, 1] + w1, l0[j, 0]:l0[j, 0] + w1] += \
            cp[j] * k[2][:, None, None] * k[1][None, :, None] * k[0][None, None, :]
    # 2. deconvolve by phi2hat, pad: mode l - n1/2 at index (l - n1/2) mod n2
    dec = [1.0 / _es_hat((np.arange(n1[d]) - n1[d] // 2) / n2[d], w2, b2) for d in range(3)]
    fine = np.zeros(tuple(n2[::-1]), complex)
    idx = [(np.arange(n1[d]) - n1[d] // 2) % n2[d] for d in range(3)]
    fine[np.ix_(idx[2], idx[1], idx[0])] = grid * dec[2][:, None, None] * dec[1][None, :, None] * dec[0][None, None, :]
    # 3. FFT
    G = np.fft.fftn(fine)
    # 4. interpolate, deconvolve by psi1hat
    qp = q - cq
    t = qp * h * n2
    p0 = np.ceil(t - w2 / 2).astype(int)
    F = np.zeros(len(q), complex)
    for k in range(len(q)):
        kv = [_es(t[k, d] - (p0[k, d] + np.arange(w2)), w2, b2) for d in range(3)]
        ii = [(p0[k, d] + np.arange(w2)) % n2[d] for d in range(3)]
        T = np.einsum("zyx,z,y,x->", G[np.ix_(ii[2], ii[1], ii[0])], kv[2], kv[1], kv[0])
        F[k] = T / np.prod([_es_hat(h[d] * qp[k, d], w1, b1)[0] for d in range(3)])
    return F


@pytest.mark.parametrize("eps", [1e-4, 1e-6, 1e-8])
def test_width_rule_meets_requested_error(eps):
    rng = np.random.Generator(np.random.PCG64(5))
    Z = rng.choice([6, 7, 8], 150).astype(np.int32)
    pos = rng.normal(size=(150, 3)) * 1e-9
    x = pos - 0.5 * (pos.min(0) + pos.max(0))
    q = O.hkl_detector(12, 10, 12 * 600e-6, 10 * 600e-6, 0.05, 0.15e-9)
    F = _nufft(x, np.ones(len(x)), q, eps)
    F64, _ = O.structure_factor(np.full(len(Z), 1, np.int32), x, q, delta_atoms=True)
    rel = np.linalg.norm(F - F64) / np.linalg.norm(F64)
    assert rel < 4 * eps, (eps, rel)
