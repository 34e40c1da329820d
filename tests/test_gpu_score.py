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
    slots = score.register(table, W)               # the same slots, passed directly
    assert slots == {n: table.add_weights(w) for n, w in W.items()}
    by_slot = score.score(table, cd, slots)
    assert all(np.array_equal(by_slot[n][1], res[n][1]) for n in W)


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


def test_weights_call_equals_single_weight_calls(setup):
    """mb_polish_peaks_weights reads the exact A/B from a device matrix; each of its rows equals
    the single-weight matrix-free call (the same A/B values, the same polish)."""
    t, cd, table = setup
    W = score.reference_weights(t.gamma)
    slots = [table.add_weights(w) for w in W.values()]
    hu, hp, dp = path1.polish_peaks_weights(table, cd, slots)
    assert hu.shape == (len(W), cd.n)
    for i, s in enumerate(slots):
        gu, gp, gd = path1.polish_peaks_exact(table, cd, s)
        np.testing.assert_allclose(hu[i], gu, rtol=0, atol=1e-15)
        np.testing.assert_allclose(hp[i], gp, rtol=0, atol=1e-15)
        np.testing.assert_allclose(dp[i], gd, rtol=0, atol=1e-15)
    hz = path1.polish_peaks_weights(table, cd, slots[:2], n_zeros=0)     # no zeros: all sums are 0
    assert np.all(hz[0] == 0.0) and np.all(hz[1] == 0.0)


def test_weights_call_in_chunks(gpu):
    """600,000 zeros: the 4 GiB matrix budget holds 447 peaks, so 460 candidates take two chunks."""
    data = synth.make_table(600_000, seed=72)
    cd = synth.make_candidates(460, seed=73)
    cd.delta[:] = np.random.default_rng(73).uniform(-1e-4, 1e-4, cd.n)
    with k2.ZeroTable.from_data(data) as table:
        w = score.reference_weights(data.gamma)["jp"]
        s = table.add_weights(w)
        hu, hp, dp = path1.polish_peaks_weights(table, cd, [s])
        gu, gp, gd = path1.polish_peaks_exact(table, cd, s)
    np.testing.assert_allclose(hu[0], gu, rtol=0, atol=1e-15)
    np.testing.assert_allclose(hp[0], gp, rtol=0, atol=1e-15)
    np.testing.assert_allclose(dp[0], gd, rtol=0, atol=1e-15)


def test_weights_call_arguments(setup):
    """mb_polish_peaks_weights rejects an empty or oversized weight list and unknown slots; no
    candidates give empty rows."""
    from mertens_bound_b200._lib import K2Error
    t, cd, table = setup
    s = table.add_weights(score.reference_weights(t.gamma)["jp"])
    with pytest.raises(K2Error):
        path1.polish_peaks_weights(table, cd, [])
    with pytest.raises(K2Error):
        path1.polish_peaks_weights(table, cd, [s] * 65)
    with pytest.raises(K2Error):
        path1.polish_peaks_weights(table, cd, [s, 999])
    hu, hp, dp = path1.polish_peaks_weights(table, cd.subset(np.arange(0)), [s, s])
    assert hu.shape == (2, 0) and hp.shape == (2, 0) and dp.shape == (2, 0)
