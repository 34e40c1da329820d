"""Grid scan against point evaluations and the oracle; the polish.py-style driver."""
from fractions import Fraction

import numpy as np
import pytest

from mertens_bound_b200 import k2, polish, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def table(gpu, small_table):
    t = k2.ZeroTable.from_data(small_table)
    yield t
    t.close()


def test_scan_matches_point_evaluations(table, small_table, oracle):
    y0 = "3484971332733132396.5383341489440461"
    step = 2e-5
    ms, h = polish.grid(table, y0, 40 * step, step, k=3e-9, T=7000.0)
    assert len(h) == 81
    vi, vf = polish.to_fixed(y0)
    si, sf = polish.to_fixed(Fraction(step))
    base, st = (vi << 64) | vf, (si << 64) | sf
    pts = [((base + int(m) * st) >> 64, (base + int(m) * st) & polish.MASK64) for m in ms]
    c = synth.Candidates(np.array([p[0] for p in pts], np.uint64), np.array([p[1] for p in pts], np.uint64),
                         np.zeros(len(pts)))
    n = small_table.count_below(7000.0)
    val, _, _ = k2.k2_plain(table, c, 3e-9, 7000.0)
    assert np.max(np.abs(h - val)) < 1e-13
    sub = c.subset(np.arange(0, 81, 10))
    hi, _ = oracle.k2(sub, small_table, 3e-9, n)
    assert np.max(np.abs(h[::10] - hi[:, 0])) < 1e-13


def test_scan_best_and_neighbours(table):
    val, yy, m = polish.scan(table, "3484971332733132396.5383341489440461", 0.01, 1e-4, k=3e-9, T=7000.0)
    ms, h = polish.grid(table, "3484971332733132396.5383341489440461", 0.01, 1e-4, k=3e-9, T=7000.0)
    assert abs(val) == np.max(np.abs(h)) and ms[np.argmax(np.abs(h))] == m
    lo, hi, v = polish.h_point(table, yy, k=3e-9, T=7000.0)
    assert lo <= v + 1e-13 and v - 1e-13 <= hi and hi - lo < 1e-11
    assert abs(v - val) < 1e-13


def test_polish_cli(gpu, capsys):
    assert polish.main(["3484971332733132396.5383341489440461", "0.001", "2e-5", "--T", "5000"]) == 0
    out = capsys.readouterr().out
    assert "GRID best" in out and "CERTIFIED" in out and "neighbor 2" in out
