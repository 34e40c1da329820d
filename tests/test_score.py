"""Host side of the candidate scoring module (no GPU)."""
import numpy as np

from mertens_bound_b200 import score, synth


def test_reference_weights():
    t = synth.make_table(20_000, seed=1)
    w = score.reference_weights(t.gamma)
    assert set(w) == {"jp", "g15", "g10", "raw", "10k"}
    assert all(v.shape == t.gamma.shape for v in w.values())
    u = t.gamma / t.gamma[-1]
    assert abs(w["jp"][-1]) < 1e-15 and abs(w["jp"][0] - ((1 - u[0]) * np.cos(np.pi * u[0]) + np.sin(np.pi * u[0]) / np.pi)) == 0
    assert w["10k"][:10_000].sum() == 10_000 and w["10k"][10_000:].sum() == 0
    assert np.all(w["g15"] <= w["g10"]) and np.all(w["raw"] == 1.0)


def test_candidates_from_x_exact():
    rng = np.random.default_rng(4)
    xs = [int(rng.integers(1 << 62)) * (1 << 30) // 7 + 12345 for _ in range(50)]
    dy = rng.uniform(-1e-4, 1e-4, 50)
    c = score.candidates_from_x(xs, dy)
    for x, vi, vf in zip(xs, c.v_int, c.v_frac):
        assert (int(vi) << 64 | int(vf)) == x << 34          # v 2^64 = x 2^34 exactly
    assert np.array_equal(c.delta, dy)
