"""Peak re-optimisation on the GPU: the contract of search/polish.py.

    python -m mertens_bound_b200.polish Y0 [HALF_WIDTH] [STEP] [--table FILE] [--k K] [--T T]

search/polish.py:75-91 evaluates h_StR(y) = 2 sum_{gamma<74000} exp(-3e-9 gamma^2) Re(c e^{i gamma y})
at y0 (256-bit mpfr), scans the FP64 grid y0 + m step for |m| <= half/step (:50-72), and
re-evaluates the best point and its +-1, +-2 neighbours in mpfr.  Here:
  * grid scan   mb_grid_scan: every grid point's phase exact (fixed-point step), FP64 sums;
  * point value the certified interval kernel ([lo, hi], rigorous) and the plain FP64 kernel.
Points are decimal strings converted to 64.64 fixed point (floor); the certified value at the
decimal point itself is obtained by widening with v_rad = 2^-64.
"""
from __future__ import annotations

import argparse
import math
import sys
from fractions import Fraction

import numpy as np

from . import k2, synth
from ._lib import check, lib, ptr

MASK64 = (1 << 64) - 1
POLISH_K, POLISH_T = 3e-9, 74000.0          # search/polish.py:14 and :28


def to_fixed(y) -> tuple[int, int]:
    """(v_int, v_frac) = floor of y (decimal string, Fraction, int or float) in 64.64."""
    f = Fraction(y) if not isinstance(y, Fraction) else y
    if f < 0 or f >= 2 ** 64:
        raise ValueError("points must lie in [0, 2^64)")
    whole = int(f)
    frac = int((f - whole) * (1 << 64))
    return whole, frac


def from_fixed(vi: int, vf: int, digits: int = 30) -> str:
    """Decimal string of v_int + v_frac 2^-64 (exact value, rounded to `digits` decimals)."""
    v = Fraction(int(vi)) + Fraction(int(vf), 1 << 64)
    q = round(v * 10 ** digits)
    s = str(q).rjust(digits + 1, "0")
    return f"{s[:-digits]}.{s[-digits:]}"


def _cands(points):
    vi = np.array([p[0] for p in points], dtype=np.uint64)
    vf = np.array([p[1] for p in points], dtype=np.uint64)
    return synth.Candidates(vi, vf, np.zeros(len(points)))


def grid(table: k2.ZeroTable, y0, half_width: float, step: float, k: float = POLISH_K, T: float = POLISH_T):
    """h on the grid y0 + m step, |m| <= round(half_width / step); returns (m values, h)."""
    m_half = int(round(half_width / step))
    si, sf = to_fixed(Fraction(step))
    vi, vf = to_fixed(y0)
    n_m = 2 * m_half + 1
    h = np.empty(n_m)
    a_int = np.array([vi], np.uint64)          # kept alive across the call
    a_frac = np.array([vf], np.uint64)
    check(lib().mb_grid_scan(table.handle, 1, ptr(a_int), ptr(a_frac), float(k), float(T), si, sf, -m_half, n_m,
                             ptr(h)))
    return np.arange(-m_half, m_half + 1), h


def scan(table: k2.ZeroTable, y0, half_width: float, step: float, k: float = POLISH_K, T: float = POLISH_T):
    """(best h, best y as a decimal string, best m) over the grid (search/polish.py:50-72)."""
    ms, h = grid(table, y0, half_width, step, k, T)
    j = int(np.argmax(np.abs(h)))
    vi, vf = to_fixed(y0)
    si, sf = to_fixed(Fraction(step))
    m = int(ms[j])
    total = ((vi << 64) | vf) + m * ((si << 64) | sf)
    return float(h[j]), from_fixed(total >> 64, total & MASK64), m


def h_point(table: k2.ZeroTable, y, k: float = POLISH_K, T: float = POLISH_T):
    """K2 at a decimal point y: (certified lo, certified hi, plain FP64 value)."""
    vi, vf = to_fixed(y)
    c = _cands([(vi, vf)])
    lo, hi, _ = k2.k2_certified(table, c, k, T, v_rad=2.0 ** -64)
    val, _, _ = k2.k2_plain(table, c, k, T)
    return float(lo[0]), float(hi[0]), float(val[0])


def _load_table(spec: str | None):
    from . import formats
    if spec is None:
        return synth.make_table_below(80_000.0, seed=1)
    if spec.endswith(".txt"):
        return formats.read_zero_cache(spec)[0]
    if spec.endswith("600k.bin"):
        return formats.table_from_fields(formats.read_zeros_600k(spec))
    return formats.table_from_fields(formats.read_zeros_bin(spec))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("y0")
    ap.add_argument("half", nargs="?", type=float, default=0.25)
    ap.add_argument("step", nargs="?", type=float, default=2e-5)
    ap.add_argument("--table", default=None, help="zero-cache .txt, zeros_600k.bin or zeros.bin (default: synthetic)")
    ap.add_argument("--k", type=float, default=POLISH_K)
    ap.add_argument("--T", type=float, default=POLISH_T)
    a = ap.parse_args(argv)
    data = _load_table(a.table)
    with k2.ZeroTable.from_data(data) as t:
        n = t.count_below(a.T)
        print(f"terms={n} g_last={data.gamma[n - 1]:.6f} half={a.half} step={a.step}", flush=True)
        lo, hi, v = h_point(t, a.y0, a.k, a.T)
        print(f"h({a.y0}) in [{lo!r}, {hi!r}] (fp64 {v!r})", flush=True)
        val, yy, m = scan(t, a.y0, a.half, a.step, a.k, a.T)
        print(f"GRID best |h| candidate h={val:.10f} y={yy} m={m}", flush=True)
        lo, hi, v = h_point(t, yy, a.k, a.T)
        print(f"CERTIFIED h in [{lo!r}, {hi!r}]", flush=True)
        si, sf = to_fixed(Fraction(a.step))
        vi, vf = to_fixed(yy)
        for d in (-2, -1, 1, 2):
            tot = ((vi << 64) | vf) + d * ((si << 64) | sf)
            lo, hi, _ = h_point(t, Fraction(tot, 1 << 64), a.k, a.T)
            print(f"  neighbor {d} h in [{lo!r}, {hi!r}]", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
