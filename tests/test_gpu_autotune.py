"""The autotuner (mb_plan_autotune + the per-workload cache) on a small plan."""
import math

import numpy as np
import pytest

from mertens_bound_b200 import autotune, k2, synth

pytestmark = pytest.mark.gpu


def test_autotune_picks_and_caches(gpu, small_table, tmp_path, monkeypatch):
    monkeypatch.setenv("MB_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    cd = synth.make_candidates(1500, seed=31)
    with k2.ZeroTable.from_data(small_table) as t, k2.Plan(t, [1000, 500], [3e-9, 1e-9], [math.inf, 20000.0]) as plan:
        ref, _, _ = plan.run(cd)
        r = autotune.autotune(plan, reps=2)
        assert not r["cached"] and tuple(r["config"]) in autotune.SPACE
        assert len(r["timings"]) == len(autotune.SPACE) and min(r["timings"].values()) == r["ms"]
        val, _, _ = plan.run(cd)
        eb = max(plan.group_info(g)["err_bound"] for g in range(2))
        assert np.max(np.abs(val - ref)) <= 2 * eb
        again = autotune.autotune(plan, reps=2)
        assert again["cached"] and tuple(again["config"]) == tuple(r["config"])
