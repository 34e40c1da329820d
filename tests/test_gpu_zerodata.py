"""The GPU leaf screen (mb_screen) and hit polish (mb_hit_scan through hit_polish.polish_hits)
against the reference enumerator's own ZeroData decisions and values, committed in
tests/golden/zerodata_ref.json (search/fast_mertens_enum.cpp:108-142 fast_screen, :145-276 polish,
compiled from the reference source; see tests/test_zerodata_ref.py for how the fixture is pinned).

The reference screen reads cos from a 16,384-entry FP32 table at a 14-bit truncated phase, with
the seven offsets rounded to table steps; the GPU sums exact-phase terms.  So decisions must agree
on every leaf whose exact score lies outside the table's error band around a threshold (per zero
at most 2.5 table steps of angle: 1 for the truncation, 1.5 for the offset rounding at m = +-3).
The polish runs the same stages on exact phases, so it must land on the same grid points and
agree in h to rounding."""
import math

import numpy as np
import pytest

from mertens_bound_b200 import hit_polish, k2
from test_zerodata_ref import ENUM_THRESHOLDS, FIX, fixture_pass, leaves, table

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gtable(gpu):
    t = table()
    zt = k2.ZeroTable.from_data(t)
    yield t, zt
    zt.close()


def test_gpu_screen_matches_reference_decisions(gtable):
    t, zt = gtable
    x, _, _ = leaves()
    pts = hit_polish.points_from_x(x)
    ends, thr = hit_polish.SCREEN_CPU
    r = hit_polish.screen_leaves(zt, pts, 3e-9, hit_polish.SCREEN_CPU, all_scores=True)
    a = 2.0 * np.hypot(t.c_re, t.c_im) * np.exp(-3e-9 * t.gamma ** 2)
    band = [float(a[:e].sum()) * 2.5 * 2 * math.pi / 16384 + 2e-5 for e in ends]
    s0, s1 = r.scores[:, 0], r.scores[:, 1]
    ref = fixture_pass().astype(bool)
    clear = np.abs(s0 - thr[0]) > band[0]
    need1 = s0 >= thr[0]
    clear &= ~need1 | (np.abs(s1 - thr[1]) > band[1])
    gpu_pass = (s0 >= thr[0]) & (s1 >= thr[1])
    assert np.array_equal(gpu_pass, np.isin(np.arange(len(x)), r.hits))
    mism = np.flatnonzero(clear & (gpu_pass != ref))
    assert mism.size == 0, (mism[:10], s0[mism[:10]], s1[mism[:10]], ref[mism[:10]])
    # the band leaves most decisions to check: both passes and failures
    assert clear.mean() > 0.9 and ref[clear].sum() > 100 and (~ref[clear]).sum() > 1000


def test_gpu_hit_polish_matches_reference(gtable):
    t, zt = gtable
    x, _, _ = leaves()
    sel = [p["leaf"] for p in FIX["polish"]]
    pts = hit_polish.points_from_x([x[i] for i in sel])
    r = hit_polish.polish_hits(zt, pts, 3e-9, thresholds=ENUM_THRESHOLDS)
    ref_h = np.array([p["h"] for p in FIX["polish"]])
    ref_dy = np.array([p["dy"] for p in FIX["polish"]])
    assert np.max(np.abs(r.dy - ref_dy)) < 1e-13, np.abs(r.dy - ref_dy)
    assert np.max(np.abs(r.h - ref_h)) < 1e-9, np.abs(r.h - ref_h)
    assert np.sum(r.stage == 4) >= 30            # most selected hits run all five stages
