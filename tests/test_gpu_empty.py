"""Empty inputs through every host entry point: no candidates, no zeros below T."""
import math

import numpy as np
import pytest

from mertens_bound_b200 import k2, path1, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def table(gpu, small_table):
    t = k2.ZeroTable.from_data(small_table.truncate(3000))
    yield t
    t.close()


def test_no_candidates(table):
    c = synth.make_candidates(4, seed=1).subset(np.arange(0))
    assert all(x.shape == (0,) for x in k2.k2_plain(table, c, 3e-9))
    assert all(x.shape == (0,) for x in k2.k2_certified(table, c, 3e-9))
    hi, lo = k2.phase128(table, c, 10)
    assert hi.shape == (0, 10)
    val, dd, dk, eb = k2.k2_fast(table, c, 3e-9)
    assert val.shape == (0,)
    with k2.Plan(table, [0], [3e-9], [math.inf]) as plan:
        assert all(x.shape == (0,) for x in plan.run(c))
        assert plan.time(1) == 0.0
    A, B = path1.compute_exact_AB(table, c, 10)
    assert A.shape == (0, 10)
    slot = table.add_weights(np.ones(table.n))
    assert all(x.shape == (0,) for x in path1.polish_peaks_exact(table, c, slot))


def test_no_zeros_below_T(table):
    c = synth.make_candidates(8, seed=2)
    val, dd, dk = k2.k2_plain(table, c, 3e-9, 1.0)
    assert np.all(val == 0) and np.all(dd == 0) and np.all(dk == 0)
    lo, hi, ab = k2.k2_certified(table, c, 3e-9, 1.0)
    assert np.all(lo <= 0) and np.all(hi >= 0) and np.all(hi - lo < 1e-300 + 1e-30)
    fv, _, _, eb = k2.k2_fast(table, c, 3e-9, 1.0)
    assert np.all(fv == 0) and eb == 0.0
