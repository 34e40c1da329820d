"""Interval (ball) oracle for K2 -- TEST INFRASTRUCTURE ONLY.

python-flint (Arb) is not installed here, so the "Arb ball" of
certification/certify_K2.py:112-121 is restated with mpmath interval arithmetic
(mpmath.iv) at a working precision of >= 200 bits:

    w = exp(-k g^2),  term = 2 w Re(c exp(i g v)),  S += term,  absS += 2 w |c|

with g = 2pi G from the exact 64.128 fixed-point G and the phase reduced exactly in
integers first (search/path1_eval_fast.cpp:45 / legacy/superseded/certify_peak2_600k.py:183),
so the interval cos/sin only ever see an argument in [0, 2pi) plus gamma delta.
This is a restatement, labelled as such; it is not python-flint.
"""
from __future__ import annotations

from fractions import Fraction

import mpmath as mp

from .oracle import phase128_bigint  # noqa: F401  (re-exported for callers)


def k2_ball(vi: int, vf: int, delta: float, G3, c_re, c_im, k: float, n_use: int, prec: int = 220):
    """Enclosures (val, dd, dk) of K2 and its derivatives as mpmath intervals."""
    iv = mp.iv
    with mp.workprec(prec):
        old = iv.prec
        iv.prec = prec
        try:
            two_pi = 2 * iv.pi
            kk = iv.mpf(float(k))
            dq = iv.mpf(float(delta))
            V = (int(vi) << 64) | int(vf)
            S = iv.mpf(0); D = iv.mpf(0); K = iv.mpf(0)
            for j in range(n_use):
                gi, g1, g2 = (int(x) for x in G3[j])
                Gf = (gi << 128) | (g1 << 64) | g2
                frac_num = (V * Gf) & ((1 << 192) - 1)            # frac(v G) 2^192, exact
                fr = iv.mpf(mp.mpf(frac_num) / mp.mpf(2) ** 192)   # exact at prec >= 192
                G = iv.mpf(mp.mpf(Gf) / mp.mpf(2) ** 128)
                g = two_pi * G
                th = two_pi * fr + g * dq
                cs, sn = iv.cos(th), iv.sin(th)
                w = iv.exp(-kk * g * g)
                cr, ci = iv.mpf(float(c_re[j])), iv.mpf(float(c_im[j]))
                re = cr * cs - ci * sn
                im = cr * sn + ci * cs
                S += w * re
                D += w * g * im
                K += w * g * g * re
            return 2 * S, -2 * D, -2 * K
        finally:
            iv.prec = old


def _exact(t) -> Fraction:
    """Exact value of an mpmath raw float tuple (sign, mantissa, exponent, bitcount)."""
    sign, man, e, _ = t
    if man == 0 and e != 0:
        raise ValueError("non-finite interval endpoint")
    v = Fraction(man) * Fraction(2) ** e
    return -v if sign else v


def bounds(x) -> tuple[Fraction, Fraction]:
    """Exact rational endpoints of an mpmath interval (read without rounding)."""
    a, b = x._mpi_
    return _exact(a), _exact(b)
