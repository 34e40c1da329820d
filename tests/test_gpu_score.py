"""Matrix-free polish_peaks_with_weights (mb_polish_peaks_exact) against the reference's own
compiled compute_peak_AB + polish_peaks_with_weights and against the A/B-matrix path."""
import numpy as np
import pytest

from mertens_bound_b200 import compat, k2, path1, score, synth
from oracle.oracle import RefLib, reference_candidates, reference_format

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(gpu, small_table):
    t = small_table.truncate(6000)
    cd = synth.make_candidates(24, seed=71)
    cd.delta[:] = np.linspace(-2e-5, 2e-5, cd.n)
    table = k2.ZeroTable.from_data(t)
    yield t, cd, table
    table.close()


def test_score_matches_matrix_path(setup):
    t, cd, table = setup
    W = score.reference_weights(t.gamma)
    res = score.score(table, cd, W)
    A, B = path1.compute_exact_AB(table, cd)
    for name, w in W.items():
        hu, hp, dp = compat.polish_peaks_with_weights(A, B, t.gamma, w, 2.5e-4, 40)
        gu, gp, gd = res[name]
        np.testing.assert_allclose(gu, hu, rtol=1e-13, atol=1e-15, err_msg=name)
        np.testing.assert_allclose(gp, hp, rtol=1e-12, atol=1e-14, err_msg=name)
        np.testing.assert_allclose(gd, dp, rtol=0, atol=1e-12, err_msg=name)
    again = score.score(table, cd, W)              # registered vectors are reused
    assert all(np.array_equal(again[n][1], res[n][1]) for n in W)


@pytest.mark.skipif(not RefLib.available(), reason="reference evaluator not built")
def test_score_matches_reference_evaluator(setup):
    t, cd, table = setup
    R = RefLib()
    A0, B0 = R.peak_AB(reference_candidates(cd), reference_format(t))
    W = score.reference_weights(t.gamma)
    res = score.score(table, cd, {"jp": W["jp"], "g10": W["g10"]})
    for name in ("jp", "g10"):
        hu0, hp0, dp0 = R.polish(A0, B0, t.gamma, W[name], 2.5e-4, 40)
        hu, hp, dp = res[name]
        assert np.max(np.abs(hu - hu0)) < 1e-12, name
        assert np.max(np.abs(hp - hp0)) < 1e-11, name
        assert np.max(np.abs(dp - dp0)) < 1e-9, name
