"""Certified interval kernel: its [lo, hi] must contain the interval oracle's ball (mpmath iv,
the restatement of certify_K2.py's Arb sum) and the binary128 value."""
import math
import time

import numpy as np
import pytest

from mertens_bound_b200 import k2, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def table(gpu, small_table):
    t = k2.ZeroTable.from_data(small_table)
    yield t
    t.close()


def test_certified_contains_interval_ball(table, small_table):
    from oracle.interval import bounds, k2_ball
    n = 1200
    cd = synth.make_candidates(3, seed=51)
    T = float(small_table.gamma[n - 1]) + 1e-9
    assert table.count_below(T) == n
    lo, hi, ab = k2.k2_certified(table, cd, 3e-9, T)
    for p in range(cd.n):
        val, _, _ = k2_ball(cd.v_int[p], cd.v_frac[p], 0.0, small_table.G3, small_table.c_re, small_table.c_im,
                            3e-9, n)
        blo, bhi = bounds(val)
        assert lo[p] <= blo and bhi <= hi[p], (lo[p], float(blo), float(bhi), hi[p])
        assert hi[p] - lo[p] < 1e-12


def test_certified_contains_quad_oracle(table, small_table, oracle):
    cd = synth.make_candidates(40, seed=52)
    for k, T in ((3e-9, math.inf), (1e-9, 20000.0), (0.0, 3000.0)):
        lo, hi, ab = k2.k2_certified(table, cd, k, T)
        ohi, olo = oracle.k2(cd, small_table, k, small_table.count_below(T))
        v = ohi[:, 0] + olo[:, 0]
        assert np.all(lo <= v) and np.all(v <= hi)
        assert np.max(hi - lo) < 1e-11
        assert np.all(ab >= np.abs(lo)) and np.all(ab >= np.abs(hi))


def test_certified_radii_widen(table):
    cd = synth.make_candidates(2, seed=53)
    lo0, hi0, _ = k2.k2_certified(table, cd, 3e-9)
    lo1, hi1, _ = k2.k2_certified(table, cd, 3e-9, v_rad=1e-12)
    assert np.all(lo1 <= lo0) and np.all(hi1 >= hi0) and np.all(hi1 - lo1 > hi0 - lo0)
    rad = np.full(table.n, 1e-9)
    lo2, hi2, _ = k2.k2_certified(table, cd, 3e-9, term_rad=rad)
    assert np.all(hi2 - lo2 > 1e-9)


def test_certified_full_peak2(gpu, oracle):
    """All 2,325,572 zeros below T0 = 1.3e6 at the reference's Peak2 point
    (certification/certify_K2.py:40-43), k = 1.5e-10, in well under a second."""
    data = synth.make_table(2_325_572, seed=1)
    cd = synth.peak2_candidate()
    with k2.ZeroTable.from_data(data) as t:
        assert t.count_below(1.3e6) == 2_325_572
        k2.k2_certified(t, cd, 1.5e-10, 1.3e6)                       # warm-up
        t0 = time.perf_counter()
        lo, hi, ab = k2.k2_certified(t, cd, 1.5e-10, 1.3e6, v_rad=2.0 ** -64)
        elapsed = time.perf_counter() - t0
    assert elapsed < 1.0
    ohi, olo = oracle.k2(cd, data, 1.5e-10, data.n)
    v = ohi[0, 0] + olo[0, 0]
    assert lo[0] <= v <= hi[0]
    assert hi[0] - lo[0] < 1e-11


def test_certified_maximum_batch(table, small_table, oracle):
    """The largest batch one call takes (65,535 points) encloses the plain FP64 values (a
    sample checked against the binary128 oracle); one more point is rejected."""
    from mertens_bound_b200._lib import K2Error
    cd = synth.make_candidates(65_535, seed=54)
    T = 2000.0
    lo, hi, _ = k2.k2_certified(table, cd, 3e-9, T)
    pv, _, _ = k2.k2_plain(table, cd, 3e-9, T)
    width = hi - lo
    assert np.max(width) < 1e-12
    assert np.all(lo - width <= pv) and np.all(pv <= hi + width)     # plain is within ~1e-15
    idx = np.arange(0, 65_535, 4_096)
    ohi, olo = oracle.k2(cd.subset(idx), small_table, 3e-9, small_table.count_below(T))
    v = ohi[:, 0] + olo[:, 0]
    assert np.all(lo[idx] <= v) and np.all(v <= hi[idx])
    with pytest.raises(K2Error, match="MB_ERR_ARG"):
        k2.k2_certified(table, synth.make_candidates(65_536, seed=55), 3e-9, T)


def test_certified_grad_contains_derivative_balls(table, small_table):
    """K2, dK2/ddelta and dK2/dk enclosures against the committed 220-bit interval balls of
    tests/golden/small_plain.json (mpmath iv, the restatement of certify_K2.py's Arb sum and its
    derivatives), and the K2 row equal to mb_k2_certified's interval."""
    import json
    import os
    from fractions import Fraction
    fx = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "small_plain.json")))
    cd = synth.make_candidates(64, seed=2).subset(np.arange(4))
    lo, hi = k2.k2_certified_grad(table, cd, fx["k"])
    vlo, vhi, _ = k2.k2_certified(table, cd, fx["k"])
    assert np.array_equal(lo[0], vlo) and np.array_equal(hi[0], vhi)
    for p in range(4):
        a, b = (Fraction(x) for x in fx["interval_balls_first4"][p])
        assert Fraction(lo[0, p]) <= a and b <= Fraction(hi[0, p])
        for row, key in ((1, "dd"), (2, "dk")):
            a, b = (Fraction(x) for x in fx["derivative_balls_first4"][p][key])
            assert Fraction(lo[row, p]) <= a and b <= Fraction(hi[row, p]), (p, key)
            mid = abs(float(a + b) / 2)
            assert hi[row, p] - lo[row, p] < 1e-10 * mid, (p, key, hi[row, p] - lo[row, p], mid)


def test_certified_grad_contains_quad_oracle(table, small_table, oracle):
    cd = synth.make_candidates(40, seed=56)
    for k, T in ((3e-9, math.inf), (1.5e-10, 30000.0)):
        lo, hi = k2.k2_certified_grad(table, cd, k, T)
        ohi, olo = oracle.k2(cd, small_table, k, small_table.count_below(T))
        for row in range(3):
            v = ohi[:, row] + olo[:, row]
            assert np.all(lo[row] <= v) and np.all(v <= hi[row]), row
        # radii widen every row
        lo2, hi2 = k2.k2_certified_grad(table, cd, k, T, v_rad=1e-12)
        assert np.all(lo2 <= lo) and np.all(hi2 >= hi) and np.all(hi2 - lo2 > hi - lo)
