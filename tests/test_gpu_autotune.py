"""The autotuner (mb_plan_autotune under both schedules + the per-workload cache) on a small plan,
and the two schedules giving the same bits."""
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
        assert not r["cached"] and tuple(r["config"][:3]) in autotune.SPACE and r["config"][3] in (0, 1, 2)
        assert len(r["timings"]) == 3 * len(autotune.SPACE) and min(r["timings"].values()) == r["ms"]
        assert plan.schedule() == r["config"][3]
        val, _, _ = plan.run(cd)
        eb = max(plan.group_info(g)["err_bound"] for g in range(2))
        assert np.max(np.abs(val - ref)) <= 2 * eb
        again = autotune.autotune(plan, reps=2)
        assert again["cached"] and tuple(again["config"]) == tuple(r["config"])


@pytest.mark.parametrize("cpt", [2, 3, 4])
def test_schedules_give_the_same_bits(gpu, small_table, cpt):
    """One persistent kernel for both tiers (in plan order or interleaved) runs the same items with
    the same per-item arithmetic as the two concurrent kernels, so every output bit agrees."""
    cd = synth.make_candidates(700, seed=32)
    cd.delta[:] = np.random.default_rng(33).uniform(-1e-4, 1e-4, cd.n)
    with k2.ZeroTable.from_data(small_table) as t, k2.Plan(t, [300, 400], [3e-9, 1.5e-10], [math.inf, 20000.0],
                                                           tol=1e-8) as plan:
        plan.configure(cpt, 0, 1.0)
        h, l = plan.tier_terms()
        assert h > 0 and l > 0                     # both tiers present
        a = plan.run(cd)
        plan.set_schedule(1)
        assert plan.schedule() == 1
        b = plan.run(cd)
        plan.set_schedule(2)
        d = plan.run(cd)
        plan.set_schedule(0)
        c = plan.run(cd)
    for x, y, z, w in zip(a, b, c, d):
        assert np.array_equal(x, y) and np.array_equal(x, z) and np.array_equal(x, w)
