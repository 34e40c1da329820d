"""Chosen form (tiered FP32/FP64 persistent kernel) against the oracle and the plain kernel."""
import math

import numpy as np
import pytest

from mertens_bound_b200 import k2, synth

pytestmark = pytest.mark.gpu

TOL = 1e-10   # |K2 error| target of the chosen form


@pytest.fixture(scope="module")
def table(gpu, small_table):
    t = k2.ZeroTable.from_data(small_table)
    yield t
    t.close()


@pytest.mark.parametrize("P", [1, 37, 64, 700, 1500])
def test_fast_vs_oracle(table, small_table, oracle, P):
    cd = synth.make_candidates(P, seed=100 + P)
    k = 3e-9
    val, dd, dk, eb = k2.k2_fast(table, cd, k, tol=TOL)
    assert eb <= TOL
    n = min(P, 64)
    ohi, _ = oracle.k2(cd.subset(np.arange(n)), small_table, k, small_table.n)
    err = np.abs(val[:n] - ohi[:, 0])
    assert np.max(err) <= eb, (np.max(err), eb)
    # gradients: same a-priori structure scaled by gamma; compare relative to their size
    assert np.max(np.abs(dd[:n] - ohi[:, 1])) <= 1e-6 * np.max(np.abs(ohi[:, 1]))
    assert np.max(np.abs(dk[:n] - ohi[:, 2])) <= 1e-6 * np.max(np.abs(ohi[:, 2]))


def test_fast_matches_plain_with_delta_and_cutoff(table):
    cd = synth.make_candidates(512, seed=7)
    cd.delta[:] = np.random.default_rng(3).uniform(-2e-4, 2e-4, 512)
    k, T = 1e-9, 20000.0
    val, dd, dk, eb = k2.k2_fast(table, cd, k, T)
    pv, pd, pk = k2.k2_plain(table, cd, k, T)
    assert np.max(np.abs(val - pv)) <= eb
    assert np.max(np.abs(dd - pd)) <= 1e-6 * np.max(np.abs(pd))


def test_batched_plan_groups(table):
    counts = [64, 300, 1024, 5]
    ks = [3e-9, 1e-9, 1.5e-10, 3e-9]
    Ts = [math.inf, 20000.0, 50000.0, 1000.0]
    P = sum(counts)
    cd = synth.make_candidates(P, seed=8)
    with k2.Plan(table, counts, ks, Ts, tol=TOL) as plan:
        assert plan.info()["light_form"] == "fused"        # every zero of the table below 3.29e6
        val, dd, dk = plan.run(cd)
        val2, _, _ = plan.run(cd)            # graph replay gives identical results
        assert np.array_equal(val, val2)
        off = 0
        for g, (c, kk, TT) in enumerate(zip(counts, ks, Ts)):
            sub = cd.subset(np.arange(off, off + c))
            pv, pd, pk = k2.k2_plain(table, sub, kk, TT)
            gi = plan.group_info(g)
            assert gi["err_bound"] <= TOL
            assert np.max(np.abs(val[off:off + c] - pv)) <= gi["err_bound"]
            off += c


def test_plan_shapes_agree(table):
    cd = synth.make_candidates(256, seed=9)
    with k2.Plan(table, [256], [3e-9], [math.inf]) as plan:
        ref, _, _ = plan.run(cd)
        eb = plan.group_info(0)["err_bound"]
        for cpt, nzw in [(2, 1), (3, 2), (4, 8), (2, 8)]:
            plan.set_shape(0, cpt, nzw, 256, 512)
            v, _, _ = plan.run(cd)
            assert np.max(np.abs(v - ref)) <= 2 * eb


def test_zero_range_shards_add_up(table):
    """Zero-range shards (one per GPU in a zero-sharded run) sum to the whole evaluation."""
    from mertens_bound_b200 import distributed
    from mertens_bound_b200._lib import check, lib
    cd = synth.make_candidates(200, seed=12)
    with k2.Plan(table, [200], [3e-9], [math.inf], tol=TOL) as plan:
        full = np.stack(plan.run(cd), axis=1)
        eb = plan.group_info(0)["err_bound"]
        parts = []
        for r in range(3):
            j0, j1 = distributed.shard_range(table.n, 3, r)
            check(lib().mb_plan_set_zero_range(plan.handle, j0, j1))
            parts.append(np.stack(plan.run(cd), axis=1))
    tot = sum(parts)
    assert np.max(np.abs(tot[:, 0] - full[:, 0])) <= 2 * eb
    assert np.max(np.abs(tot[:, 1] - full[:, 1])) <= 1e-9 * np.max(np.abs(full[:, 1]))


def test_all_heavy_when_tolerance_tight(table, small_table, oracle):
    cd = synth.make_candidates(16, seed=10)
    with k2.Plan(table, [16], [3e-9], [math.inf], tol=1e-14) as plan:
        gi = plan.group_info(0)
        assert gi["n_heavy"] == gi["n_T"]
        val, _, _ = plan.run(cd)
    ohi, _ = oracle.k2(cd, small_table, 3e-9, small_table.n)
    assert np.max(np.abs(val - ohi[:, 0])) < 1e-12


def test_tail_skip_within_bound(gpu, oracle):
    """Skipping the negligible tail keeps |K2 - oracle| within the plan's bound (which now
    includes the skipped sum) and evaluates fewer zeros."""
    data = synth.make_table(60_000, seed=6)
    cd = synth.make_candidates(96, seed=61)
    k = 1e-8      # the Gaussian makes the zeros above gamma ~ 3e4 negligible at 1e-10
    ohi, _ = oracle.k2(cd, data, k, data.n)
    with k2.ZeroTable.from_data(data) as t, k2.Plan(t, [96], [k], [math.inf], tol=TOL) as plan:
        full, _, _ = plan.run(cd)
        plan.set_skip(0.25)
        gi = plan.group_info(0)
        assert gi["n_eval"] < gi["n_T"] == data.n
        assert gi["err_bound"] <= TOL
        val, _, _ = plan.run(cd)
        assert np.max(np.abs(val - ohi[:, 0])) <= gi["err_bound"]
        plan.set_skip(0.0)
        assert plan.group_info(0)["n_eval"] == data.n
        again, _, _ = plan.run(cd)
        assert np.array_equal(again, full)


def test_plan_ragged_and_empty_groups(table, small_table):
    """Groups with no candidates, with no zeros below T (the sum is 0), and with one candidate."""
    counts = [0, 17, 0, 33, 1, 5]
    ks = [3e-9, 1e-9, 3e-9, 3e-9, 1.5e-10, 3e-9]
    Ts = [math.inf, 5000.0, 100.0, 10.0, math.inf, 14.0]     # gamma_1 ~ 14.13: T = 10, 14 keep none
    cd = synth.make_candidates(sum(counts), seed=12)
    with k2.Plan(table, counts, ks, Ts, tol=TOL) as plan:
        val, dd, dk = plan.run(cd)
        off = 0
        for g, (c, kk, TT) in enumerate(zip(counts, ks, Ts)):
            if c == 0:
                continue
            sub = cd.subset(np.arange(off, off + c))
            pv, _, _ = k2.k2_plain(table, sub, kk, TT)
            gi = plan.group_info(g)
            if gi["n_T"] == 0:
                assert np.all(val[off:off + c] == 0) and np.all(pv == 0)
            assert np.max(np.abs(val[off:off + c] - pv)) <= gi["err_bound"] + 1e-15
            off += c


@pytest.mark.parametrize("k,skip", [(3e-9, 0.0), (1e-9, 0.0), (1e-8, 0.25)])
def test_derivative_bounds(table, small_table, oracle, k, skip):
    """K2, dK2/ddelta and dK2/dk each within their plan's a-priori bound of the oracle."""
    cd = synth.make_candidates(64, seed=13)
    cd.delta[:] = np.random.default_rng(14).uniform(-1e-4, 1e-4, 64)
    ohi, _ = oracle.k2(cd, small_table, k, small_table.n)
    with k2.Plan(table, [64], [k], [math.inf], tol=TOL) as plan:
        plan.set_skip(skip)
        val, dd, dk = plan.run(cd)
        gi = plan.group_info(0)
    assert gi["err_bound"] <= TOL
    for got, q, key in ((val, 0, "err_bound"), (dd, 1, "err_bound_dd"), (dk, 2, "err_bound_dk")):
        assert np.max(np.abs(got - ohi[:, q])) <= gi[key], key
    # the derivative bounds scale with gamma and gamma^2 of the zeros that matter
    assert gi["err_bound"] < gi["err_bound_dd"] < gi["err_bound_dk"]


def test_table_outlives_its_plans(gpu, small_table):
    """The library refuses to free a table under a live plan; the Python table closes its plans."""
    from mertens_bound_b200._lib import lib
    t = k2.ZeroTable.from_data(small_table.truncate(2000))
    plan = k2.Plan(t, [8], [3e-9], [math.inf])
    assert lib().mb_table_destroy(t.handle) == -5          # MB_ERR_STATE
    assert "plan" in lib().mb_last_error().decode()
    plan.run(synth.make_candidates(8, seed=1))             # the table is intact
    t.close()
    with pytest.raises(ValueError):
        plan.handle


def test_shards_with_skip_and_weights(gpu, oracle):
    """Zero-range shards of a plan with a tail skip and a mix of weight vectors add up to the
    unsharded run, and each group stays within its bound of the oracle."""
    from mertens_bound_b200 import distributed, score
    from mertens_bound_b200._lib import check, lib
    data = synth.make_table(40_000, seed=8)
    cd = synth.make_candidates(96, seed=81)
    W = score.reference_weights(data.gamma)
    with k2.ZeroTable.from_data(data) as t:
        slots = [t.add_weights(W["jp"]), -1, t.add_weights(W["g15"])]
        with k2.Plan(t, [32, 32, 32], [0.0, 1e-8, 0.0], [math.inf, math.inf, 20000.0], tol=TOL,
                     weights=slots) as plan:
            plan.set_skip(0.25)
            full = np.stack(plan.run(cd), axis=1)
            bounds = [plan.group_info(g) for g in range(3)]
            parts = []
            for r in range(4):
                j0, j1 = distributed.shard_range(t.n, 4, r)
                check(lib().mb_plan_set_zero_range(plan.handle, j0, j1))
                parts.append(np.stack(plan.run(cd), axis=1))
    tot = sum(parts)
    for g, (w, k, T) in enumerate(((W["jp"], 0.0, math.inf), (None, 1e-8, math.inf), (W["g15"], 0.0, 20000.0))):
        sl = slice(32 * g, 32 * g + 32)
        n = data.count_below(T)
        ohi, _ = oracle.k2(cd.subset(np.arange(32 * g, 32 * g + 32)), data, k, n, weights=w)
        assert np.max(np.abs(full[sl, 0] - ohi[:, 0])) <= bounds[g]["err_bound"]
        assert np.max(np.abs(tot[sl, 0] - full[sl, 0])) <= 2 * bounds[g]["err_bound"]


@pytest.mark.parametrize("tol", [1e-6, 1e-7, 1e-8])
def test_high_gamma_table(gpu, small_table, oracle, tol):
    """A table of 3,000 zeros above gamma = 5e6: G's integer part exceeds 2^19, so the light tier
    takes its split fraction product (the one-FMA form needs gamma < 3.29e6).  Raw weights (k = 0)
    and the coefficients of zeros 7,000-9,999 of the small table: tol 1e-6 puts every zero in the
    light tier, 1e-7 about two thirds in the heavy one, 1e-8 nearly all."""
    rng = np.random.default_rng(91)
    gam = 5.0e6 + np.cumsum(rng.uniform(0.2, 0.72, 3000))
    G3 = synth.fixed_from_double(gam / (2.0 * math.pi), rng)
    data = synth.ZeroTableData(G3, synth.gamma_from_fixed(G3), small_table.c_re[7000:10000].copy(),
                               small_table.c_im[7000:10000].copy(), small_table.seed)
    cd = synth.make_candidates(64, seed=92)
    ohi, _ = oracle.k2(cd, data, 0.0, data.n)
    with k2.ZeroTable.from_data(data) as t:
        val, dd, dk, eb = k2.k2_fast(t, cd, 0.0, tol=tol)
        with k2.Plan(t, [64], [0.0], [math.inf], tol=tol) as plan:
            gi = plan.group_info(0)
            assert plan.info()["light_form"] == "split"
    assert gi["n_heavy"] < data.n and (gi["n_heavy"] > 0) == (tol < 1e-6)
    assert eb <= tol
    assert np.max(np.abs(val - ohi[:, 0])) <= eb
    assert np.max(np.abs(dd - ohi[:, 1])) <= gi["err_bound_dd"]
    assert np.max(np.abs(dk - ohi[:, 2])) <= gi["err_bound_dk"]
