"""The autotuner (mb_plan_autotune under every schedule + the per-workload cache) on a small plan,
and the schedules giving the same bits."""
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
        assert not r["cached"] and tuple(r["config"][:3]) in autotune.SPACE and r["config"][3] in autotune.SCHEDULES
        assert autotune.SCHEDULES == (0, 1, 2, 3)
        assert len(r["timings"]) == len(autotune.SCHEDULES) * len(autotune.SPACE)
        assert min(r["timings"].values()) == r["ms"]
        assert plan.schedule() == r["config"][3]
        val, _, _ = plan.run(cd)
        eb = max(plan.group_info(g)["err_bound"] for g in range(2))
        assert np.max(np.abs(val - ref)) <= 2 * eb
        again = autotune.autotune(plan, reps=2)
        assert again["cached"] and tuple(again["config"]) == tuple(r["config"])


@pytest.mark.parametrize("cpt", [2, 3, 4])
def test_schedules_give_the_same_bits(gpu, small_table, cpt):
    """One persistent kernel for both tiers (in plan order, interleaved, or one CTA of each tier per
    SM) runs the same items with the same per-item arithmetic as the two concurrent kernels, so
    every output bit agrees."""
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
        plan.set_schedule(3)
        e = plan.run(cd)
        plan.set_schedule(0)
        c = plan.run(cd)
    for x, y, z, w, u in zip(a, b, c, d, e):
        assert np.array_equal(x, y) and np.array_equal(x, z) and np.array_equal(x, w) and np.array_equal(x, u)


def test_one_tier_runs_in_every_schedule(gpu, small_table):
    """mb_plan_run_tiers_dev with one tier gives that tier's terms only, whatever the schedule (the
    cost-ordered schedule keeps its own item list for the one-kernel run)."""
    import torch
    from mertens_bound_b200._lib import check, lib
    dev = torch.device("cuda", 0)
    cd = synth.make_candidates(600, seed=35)
    vi = torch.from_numpy(cd.v_int.view(np.int64).copy()).to(dev)
    vf = torch.from_numpy(cd.v_frac.view(np.int64).copy()).to(dev)
    out = torch.empty(3, 3, 600, dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    res = {}
    with k2.ZeroTable.from_data(small_table) as t, k2.Plan(t, [600], [3e-9], [math.inf], tol=1e-8) as plan:
        for sched in (0, 1, 2, 3):
            plan.set_schedule(sched)
            for i, tiers in enumerate((1, 2, 3)):
                o = out[i]
                check(lib().mb_plan_run_tiers_dev(plan.handle, tiers, vi.data_ptr(), vf.data_ptr(), None,
                                                  o[0].data_ptr(), o[1].data_ptr(), o[2].data_ptr(), s))
            torch.cuda.synchronize(dev)
            res[sched] = out.cpu().numpy().copy()
        eb = plan.group_info(0)["err_bound"]
    for sched in (1, 2, 3):
        assert np.array_equal(res[sched], res[0])
    o = res[0]
    assert np.max(np.abs(o[0, 0] + o[1, 0] - o[2, 0])) <= 1e-3 * eb


def test_kernel_timing_hook(gpu, small_table):
    """mb_plan_kernel_timing / mb_plan_kernel_times: per-run tier kernel durations under each
    schedule (one launch under the one-kernel schedules, reported as the light time)."""
    import ctypes as C

    import torch
    from mertens_bound_b200._lib import check, lib
    L = lib()
    dev = torch.device("cuda", 0)
    cd = synth.make_candidates(512, seed=34)
    vi = torch.from_numpy(cd.v_int.view(np.int64).copy()).to(dev)
    vf = torch.from_numpy(cd.v_frac.view(np.int64).copy()).to(dev)
    out = torch.empty(3, 512, dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    with k2.ZeroTable.from_data(small_table) as t, k2.Plan(t, [512], [3e-9], [math.inf], tol=1e-8) as plan:
        for sched in (0, 1, 2, 3):
            plan.set_schedule(sched)
            check(L.mb_plan_kernel_timing(plan.handle, 4))
            for tiers in (3, 3, 1, 2):
                check(L.mb_plan_run_tiers_dev(plan.handle, tiers, vi.data_ptr(), vf.data_ptr(), None,
                                              out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), s))
            lt, ht, n = (C.c_double * 4)(), (C.c_double * 4)(), C.c_int()
            check(L.mb_plan_kernel_times(plan.handle, 4, lt, ht, C.byref(n)))
            assert n.value == 4
            both_heavy = [ht[0], ht[1]]
            assert all(x > 0 for x in (lt[0], lt[1], ht[2], lt[3]))
            assert ht[3] == -1 and lt[2] == -1
            if sched == 0:
                assert all(x > 0 for x in both_heavy)
            else:
                assert all(x == -1 for x in both_heavy)
            check(L.mb_plan_kernel_timing(plan.handle, 0))


def test_schedule_argument_checks(gpu, small_table):
    """mb_plan_set_schedule accepts 0..3 and rejects anything else without changing the plan."""
    from mertens_bound_b200._lib import K2Error
    cd = synth.make_candidates(200, seed=36)
    with k2.ZeroTable.from_data(small_table) as t, k2.Plan(t, [200], [3e-9], [math.inf], tol=1e-8) as plan:
        ref = plan.run(cd)
        plan.set_schedule(3)
        for bad in (-1, 4, 7):
            with pytest.raises(K2Error):
                plan.set_schedule(bad)
        assert plan.schedule() == 3
        for x, y in zip(plan.run(cd), ref):
            assert np.array_equal(x, y)
