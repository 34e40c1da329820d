"""Writes poly_coeffs.h: polynomial coefficients for the sine/cosine evaluations of the
K2 kernels, fitted here from the mathematics (Chebyshev interpolation in mpmath at 60
digits, coefficients rounded to the target type).  Run: python gen_poly.py > poly_coeffs.h

All polynomials are in the *turn* variable (angle = 2 pi t or pi t) so the kernels never
multiply the exactly reduced phase by an inexact 2 pi before the polynomial.

  HALF_S(u), HALF_C(u):  sin(pi t) = t * HALF_S(t^2),  cos(pi t) = HALF_C(t^2),  |t| <= 1/2
  QUAD_S(u), QUAD_C(u):  sin(2 pi r) = r * QUAD_S(r^2), cos(2 pi r) = QUAD_C(r^2), |r| <= 1/8
  F32_S(u),  F32_C(u):   the same quarter-turn pair in binary32, |r| <= 1/8
"""
import sys

import mpmath as mp

mp.mp.dps = 60


def fit(f, a, b, deg, relative=True):
    """Polynomial p (ascending coefficients) of degree deg interpolating f at Chebyshev
    nodes of [a, b]; returns (coeffs, max relative (or absolute) error on a dense grid)."""
    n = deg + 1
    xs = [(a + b) / 2 + (b - a) / 2 * mp.cos(mp.pi * (2 * i + 1) / (2 * n)) for i in range(n)]
    A = mp.matrix([[x ** j for j in range(n)] for x in xs])
    y = mp.matrix([f(x) for x in xs])
    c = mp.lu_solve(A, y)
    coeffs = [c[j] for j in range(n)]
    err = 0
    for i in range(2001):
        x = a + (b - a) * i / 2000
        p = sum(coeffs[j] * x ** j for j in range(n))
        fx = f(x)
        err = max(err, abs((p - fx) / fx) if relative else abs(p - fx))
    return coeffs, err


def emit(name, coeffs, ctype, fmt):
    vals = ", ".join(fmt(c) for c in coeffs)
    return f"static __device__ __constant__ const {ctype} {name}[{len(coeffs)}] = {{{vals}}};"


def f64(c):
    return repr(float(c))


def f32(c):
    import numpy as np
    return repr(float(np.float32(float(c)))) + "f"


def main():
    out = ["// Generated by gen_poly.py -- polynomial coefficients fitted by Chebyshev interpolation.",
           "// Ascending powers of u = t^2; see gen_poly.py for the meaning of each set.",
           "#pragma once"]
    sets = [
        ("HALF_S", lambda u: mp.sin(mp.pi * mp.sqrt(u)) / mp.sqrt(u) if u > 0 else mp.pi, mp.mpf(0), mp.mpf(1) / 4, 8, "double", f64),
        ("HALF_C", lambda u: mp.cos(mp.pi * mp.sqrt(u)), mp.mpf(0), mp.mpf(1) / 4, 9, "double", f64),
        ("QUAD_S", lambda u: mp.sin(2 * mp.pi * mp.sqrt(u)) / mp.sqrt(u) if u > 0 else 2 * mp.pi, mp.mpf(0), mp.mpf(1) / 64, 5, "double", f64),
        ("QUAD_C", lambda u: mp.cos(2 * mp.pi * mp.sqrt(u)), mp.mpf(0), mp.mpf(1) / 64, 5, "double", f64),
        ("F32_S", lambda u: mp.sin(2 * mp.pi * mp.sqrt(u)) / mp.sqrt(u) if u > 0 else 2 * mp.pi, mp.mpf(0), mp.mpf(1) / 64, 3, "float", f32),
        ("F32_C", lambda u: mp.cos(2 * mp.pi * mp.sqrt(u)), mp.mpf(0), mp.mpf(1) / 64, 4, "float", f32),
    ]
    for name, f, a, b, deg, ctype, fmt in sets:
        rel = name.endswith("_S")
        c, err = fit(f, a, b, deg, relative=rel)
        kind = "rel." if rel else "abs."
        out.append(f"// {name}: degree {deg} in u, max {kind} fit error {mp.nstr(err, 3)}")
        out.append(emit(name, c, ctype, fmt))
    out += certified_sets()
    print("\n".join(out))


def outward(q):
    """Doubles (lo, hi) with lo <= q <= hi for an exact rational q."""
    import math
    from fractions import Fraction
    d = float(q)
    lo = d if Fraction(d) <= q else math.nextafter(d, -math.inf)
    hi = d if Fraction(d) >= q else math.nextafter(d, math.inf)
    return lo, hi


def certified_sets():
    """Taylor coefficients of sin x / x and cos x in u = x^2 as outward-rounded intervals
    (exact rationals (-1)^k/(2k+1)! and (-1)^k/(2k)!), and an enclosure of pi/2, for the
    directed-rounding interval kernel.  Used on 0 <= x <= pi/4 with the Lagrange remainder
    x^19/19! (sine, 9 terms) and x^20/20! (cosine, 10 terms) added separately."""
    import math
    from fractions import Fraction
    s = [Fraction((-1) ** k, math.factorial(2 * k + 1)) for k in range(9)]
    c = [Fraction((-1) ** k, math.factorial(2 * k)) for k in range(10)]
    out = ["// CERT_*: exact Taylor coefficients rounded outward (lo <= exact <= hi)"]
    for name, q in (("CERT_S", s), ("CERT_C", c)):
        lo, hi = zip(*(outward(x) for x in q))
        out.append(f"static __device__ __constant__ const double {name}_LO[{len(q)}] = {{{', '.join(repr(x) for x in lo)}}};")
        out.append(f"static __device__ __constant__ const double {name}_HI[{len(q)}] = {{{', '.join(repr(x) for x in hi)}}};")
    with mp.workprec(300):
        pio2 = mp.pi / 2
        num, den = (pio2 * mp.mpf(2) ** 300), mp.mpf(2) ** 300
        q = Fraction(int(mp.floor(num)), int(den))
        lo, _ = outward(q)
        _, hi = outward(q + Fraction(1, int(den)))
    out.append(f"#define CERT_PIO2_LO {lo!r}")
    out.append(f"#define CERT_PIO2_HI {hi!r}")
    out.append(f"#define CERT_REM_S {outward(Fraction(1, math.factorial(19)))[1]!r}   // 1/19! rounded up")
    out.append(f"#define CERT_REM_C {outward(Fraction(1, math.factorial(20)))[1]!r}   // 1/20! rounded up")
    return out


if __name__ == "__main__":
    sys.exit(main())
