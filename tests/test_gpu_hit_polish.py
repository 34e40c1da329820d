"""Staged hit polish (ZeroData::polish on the GPU) against the oracle's numpy restatement."""
import numpy as np
import pytest

from mertens_bound_b200 import hit_polish, k2, synth
from oracle.oracle import Oracle, reference_format, zerodata_polish

pytestmark = pytest.mark.gpu


def test_hit_polish_matches_restated_reference(gpu):
    data = synth.make_table(20_000, seed=41)
    rng = np.random.default_rng(5)
    xs = [int(rng.integers(3_400_000_000_000_000_000, 3_600_000_000_000_000_000)) << 30 |
          int(rng.integers(0, 1 << 30)) for _ in range(6)]
    pts = hit_polish.points_from_x(xs)
    with k2.ZeroTable.from_data(data) as t:
        res = hit_polish.polish_hits(t, pts, thresholds=(None, None, None))      # run all 5 stages
        res_default = hit_polish.polish_hits(t, pts)
    assert np.all(res.stage == 4)
    reft = reference_format(data, exact_psi=True)
    two_astar = 2 * reft["alpha"] * np.exp(-3e-9 * data.gamma ** 2)
    O = Oracle()
    x_lo = np.array([x & ((1 << 64) - 1) for x in xs], np.uint64)
    x_hi = np.array([x >> 64 for x in xs], np.uint64)
    A, B, top = O.ref_peak_AB((x_lo, x_hi, np.zeros(6)), reft, want_top=True)
    for i in range(6):
        h, dy = zerodata_polish(top[i].view(np.int64), two_astar, data.gamma, thresholds=(None, None, None))
        assert abs(res.h[i] - h) < 1e-11 * max(1.0, abs(h))
        assert abs(res.dy[i] - dy) < 1e-12
        hd, dyd = zerodata_polish(top[i].view(np.int64), two_astar, data.gamma)
        assert abs(res_default.h[i] - hd) < 1e-11 and abs(res_default.dy[i] - dyd) < 1e-12
