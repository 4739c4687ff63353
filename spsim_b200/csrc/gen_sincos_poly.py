"""Generate ``sincos_poly.h``: minimax polynomials for sin(2*pi*y) and cos(2*pi*y)
in *cycles* y, used by the accurate FP32 structure-factor kernel on the FMA pipe.

Method: Remez exchange (E. Remez, 1934) on a dense grid, in the variable
z = y^2, minimising the absolute error of
    S(y) = y * P(z)  ~  sin(2 pi y)      (weight sqrt(z) on P - sin(2 pi sqrt z)/sqrt z)
    C(y) = Q(z)      ~  cos(2 pi y)
over |y| <= Y.  Coefficients are then rounded to float32 and the error of the
float32 Horner evaluation (with fused multiply-add, as the kernel does it) is
measured and printed into the header.  No library sin/cos internals are used:
the reference values come from numpy's float64 sin/cos.

The domains generated:
  HALF:  |y| <= 1/4 + 1/16  (half-cycle reduction plus the phase cross-term)
  QUAD:  |y| <= 1/8 + 1/16  (quarter-cycle reduction plus the cross-term)
  DHALF: |y| <= 1/4         (half-cycle reduction of an FP64 phase, no cross-term)
  WIDE:  |y| <= 3/8         (the second pixel of a neighbour pair: DHALF plus a
                             step of at most 1/8 cycle)
  NARROW: |y| <= 0.32       (the same where every step is at most 0.07 cycle:
                             one sine coefficient fewer at WIDE's accuracy)
  WIDER: |y| <= 0.41        (the pixels of a neighbour quad two steps from the
                             anchor: DHALF plus a step of at most 0.16 cycle;
                             WIDE's degrees at WIDE's accuracy)
Degrees are the smallest whose float32 evaluation stays near the float32
rounding floor (a higher sine degree on HALF only adds rounding error).

Usage: python gen_sincos_poly.py > sincos_poly.h
"""
import numpy as np


def remez(f, w, a, b, deg, iters=60, ngrid=40000):
    """Weighted minimax polynomial of degree ``deg`` for f on [a, b] (float64)."""
    xs = np.linspace(a, b, ngrid)
    fx, wx = f(xs), w(xs)
    n = deg + 2
    # initial reference: Chebyshev extrema mapped to [a, b]
    k = np.arange(n)
    ref = (a + b) / 2 + (b - a) / 2 * np.cos(np.pi * k / (n - 1))[::-1]
    ref = np.array([xs[np.argmin(np.abs(xs - r))] for r in ref])
    coeffs = None
    for _ in range(iters):
        A = np.zeros((n, n))
        for i, x in enumerate(ref):
            A[i, : deg + 1] = x ** np.arange(deg + 1)
            A[i, deg + 1] = (-1) ** i / w(np.array([x]))[0]
        sol = np.linalg.solve(A, f(ref))
        coeffs = sol[: deg + 1]
        err = (np.polyval(coeffs[::-1], xs) - fx) * wx
        # new reference: alternating extrema of the error
        sign = np.sign(err)
        sign[sign == 0] = 1
        idx, start = [], 0
        for i in range(1, ngrid + 1):
            if i == ngrid or sign[i] != sign[start]:
                seg = np.arange(start, i)
                idx.append(seg[np.argmax(np.abs(err[seg]))])
                start = i
        idx = np.array(idx)
        while len(idx) > n:  # drop the smallest end extremum
            if abs(err[idx[0]]) < abs(err[idx[-1]]):
                idx = idx[1:]
            else:
                idx = idx[:-1]
        if len(idx) < n:
            break
        new_ref = xs[idx]
        if np.allclose(new_ref, ref):
            break
        ref = new_ref
    return coeffs


def f32_horner(coeffs32, z32):
    """Horner with a float32 fused multiply-add per step (product exact in float64)."""
    p = np.full_like(z32, coeffs32[-1])
    for c in coeffs32[-2::-1]:
        p = (p.astype(np.float64) * z32.astype(np.float64) + np.float64(c)).astype(np.float32)
    return p


def fit(Y, sdeg, cdeg):
    """Constant terms pinned: S_0 = float32(2 pi) and C_0 = 1, so phases near
    zero (the bright forward-scattering pixels, where every atom's phase is
    small) keep float32 relative accuracy; Remez fits the remaining
    coefficients for the absolute error of sin and cos."""
    z_hi = Y * Y
    z_lo = z_hi * 1e-7  # keeps the vanishing weights below off zero
    s0 = np.float64(np.float32(2 * np.pi))
    # sin: P(z) = s0 + z P1(z) ~ sin(2 pi sqrt z)/sqrt z; the error of sin is sqrt(z) z (P1 - g)
    gs = lambda z: (np.sin(2 * np.pi * np.sqrt(z)) / np.sqrt(z) - s0) / z
    ws = lambda z: z ** 1.5
    # cos: Q(z) = 1 + z Q1(z); the error of cos is z (Q1 - g)
    gc = lambda z: (np.cos(2 * np.pi * np.sqrt(z)) - 1.0) / z
    wc = lambda z: z
    ps = np.concatenate([[s0], remez(gs, ws, z_lo, z_hi, sdeg - 1)])
    pc = np.concatenate([[1.0], remez(gc, wc, z_lo, z_hi, cdeg - 1)])
    ps32 = ps.astype(np.float32)
    pc32 = pc.astype(np.float32)
    y = np.linspace(-Y, Y, 400001).astype(np.float32)
    z = (y.astype(np.float64) * y.astype(np.float64)).astype(np.float32)
    S = (y.astype(np.float64) * f32_horner(ps32, z).astype(np.float64)).astype(np.float32)
    C = f32_horner(pc32, z)
    es = np.max(np.abs(S.astype(np.float64) - np.sin(2 * np.pi * y.astype(np.float64))))
    ec = np.max(np.abs(C.astype(np.float64) - np.cos(2 * np.pi * y.astype(np.float64))))
    rs = np.sqrt(np.mean((S.astype(np.float64) - np.sin(2 * np.pi * y.astype(np.float64))) ** 2))
    rc = np.sqrt(np.mean((C.astype(np.float64) - np.cos(2 * np.pi * y.astype(np.float64))) ** 2))
    return ps32, pc32, es, ec, rs, rc


def emit(name, Y, sdeg, cdeg, out):
    ps32, pc32, es, ec, rs, rc = fit(Y, sdeg, cdeg)
    out.append("/* %s: |y| <= %.6f cycles; float32 evaluation error vs float64:" % (name, Y))
    out.append(" *   sin max %.3e rms %.3e, cos max %.3e rms %.3e */" % (es, rs, ec, rc))
    out.append("#define SPSIM_%s_YMAX %.9ef" % (name, Y))
    out.append("#define SPSIM_%s_SIN_DEG %d" % (name, len(ps32)))
    out.append("#define SPSIM_%s_COS_DEG %d" % (name, len(pc32)))
    for k, c in enumerate(ps32):
        out.append("#define SPSIM_%s_S%d %.9ef" % (name, k, c))
    for k, c in enumerate(pc32):
        out.append("#define SPSIM_%s_C%d %.9ef" % (name, k, c))


def main():
    out = [
        "/* Generated by gen_sincos_poly.py (Remez minimax, float32 coefficients).",
        " * sin(2 pi y) ~ y * sum_k S_k (y^2)^k,  cos(2 pi y) ~ sum_k C_k (y^2)^k. */",
        "#ifndef SPSIM_B200_SINCOS_POLY_H",
        "#define SPSIM_B200_SINCOS_POLY_H",
    ]
    emit("HALF", 0.25 + 1.0 / 16, 4, 5, out)
    emit("QUAD", 0.125 + 1.0 / 16, 4, 4, out)
    emit("DHALF", 0.25, 4, 4, out)
    emit("WIDE", 0.375, 5, 5, out)
    emit("NARROW", 0.32, 4, 5, out)
    emit("WIDER", 0.41, 5, 5, out)
    out += ["#endif", ""]
    print("\n".join(out))


if __name__ == "__main__":
    main()
