"""The chosen form against the binary128 oracle at the workload sizes it is measured on.

* search scoring: all 466,659 zeros below T0 = 3e5, 4,096 candidates, k = 3e-9, tol = 1e-10 --
  the bench step, where the light tier carries most of the zeros; the first 64 candidates are
  checked at every light-kernel tile width.
* batched uneven: 16,384 candidates in 12 groups over T in {1e5, 3e5, 6e5, 1.3e6} x k in
  {3e-9, 1e-9, 1.5e-10}, one plan over the 2,325,572-zero table; four candidates per group.
* Newton polish: 1,024 candidates at T0 = 1.3e6, k = 1.5e-10 with exact 64.64 bases and FP64
  offsets delta; K2, dK2/ddelta and dK2/dk of 16 candidates, the delta-step-1e-4 central
  difference of 8, and 8 batched Newton steps.

Each output is held to its plan's a-priori bound (mb_plan_group_bounds).  The sums being checked
restate search/path1_eval_fast.cpp:35-50 (exact phase, angle, cos/sin) and :76-81 (h0 = sum w A),
with certification/certify_K2.py:116-121's term 2 w Re(c e^{i gamma v}).
"""
import math

import numpy as np
import pytest

from mertens_bound_b200 import k2, synth

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _check_bounds(plan, g, got, ohi, rows=None):
    """val, dd, dk (each (n,)) against the oracle's (n, 3) within group g's bounds."""
    gi = plan.group_info(g)
    for q, key in ((0, "err_bound"), (1, "err_bound_dd"), (2, "err_bound_dk")):
        err = np.max(np.abs(got[q] - ohi[:, q]))
        assert err <= gi[key], (g, key, err, gi[key])
    return gi


@pytest.fixture(scope="module")
def scoring(gpu, oracle):
    data = synth.make_table_below(3e5, seed=1)
    cands = synth.make_candidates(4096, seed=3)
    n_T = data.count_below(3e5)
    ohi, _ = oracle.k2(cands.subset(np.arange(64)), data, 3e-9, n_T)
    t = k2.ZeroTable.from_data(data)
    yield data, cands, t, ohi
    t.close()


def test_search_scoring_light_tier_vs_oracle(scoring):
    data, cands, t, ohi = scoring
    with k2.Plan(t, [4096], [3e-9], [3e5], tol=TOL) as plan:
        gi = plan.group_info(0)
        assert gi["n_T"] == 466_659
        # the light tier carries the bulk of the zeros at this size
        assert gi["n_heavy"] < 0.15 * gi["n_T"], gi
        assert gi["err_bound"] <= TOL
        assert plan.info()["light_form"] == "fused"
        first = None
        for cpt in (2, 3, 4):
            plan.configure(cpt, 0, 1.0)
            val, dd, dk = plan.run(cands)
            got = np.stack([val[:64], dd[:64], dk[:64]])
            _check_bounds(plan, 0, got, ohi)
            if first is None:
                first = val
            else:            # the tile width regroups the FP32 sums only: well inside the bound
                assert np.max(np.abs(val - first)) <= 2 * gi["err_bound"]
        # the one-kernel schedules (heavy first, by cost, one queue per tier) give the same bits
        # as the two concurrent kernels at this size
        last = (val, dd, dk)
        for sched in (1, 2, 3):
            plan.set_schedule(sched)
            for x, y in zip(plan.run(cands), last):
                assert np.array_equal(x, y), sched


def test_search_scoring_split_tiers_add_up(scoring):
    """The heavy tier alone plus the light tier alone is the full step (device-pointer runs)."""
    import torch
    from mertens_bound_b200._lib import check, lib
    data, cands, t, ohi = scoring
    dev = torch.device("cuda", 0)
    vi = torch.from_numpy(cands.v_int.view(np.int64).copy()).to(dev)
    vf = torch.from_numpy(cands.v_frac.view(np.int64).copy()).to(dev)
    dl = torch.zeros(4096, dtype=torch.float64, device=dev)
    outs = torch.empty(3, 3, 4096, dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    with k2.Plan(t, [4096], [3e-9], [3e5], tol=TOL) as plan:
        for i, tiers in enumerate((1, 2, 3)):
            o = outs[i]
            check(lib().mb_plan_run_tiers_dev(plan.handle, tiers, vi.data_ptr(), vf.data_ptr(), dl.data_ptr(),
                                              o[0].data_ptr(), o[1].data_ptr(), o[2].data_ptr(), s))
        torch.cuda.synchronize(dev)
        eb = plan.group_info(0)["err_bound"]
    o = outs.cpu().numpy()
    assert np.max(np.abs(o[0, 0] + o[1, 0] - o[2, 0])) <= 1e-3 * eb
    assert np.max(np.abs(o[2, 0, :64] - ohi[:, 0])) <= eb


@pytest.fixture(scope="module")
def big(gpu):
    data = synth.make_table(2_325_572, seed=1)
    t = k2.ZeroTable.from_data(data)
    yield data, t
    t.close()


def test_batched_uneven_groups_vs_oracle(big, oracle):
    data, t = big
    counts, ks, Ts = synth.batched_uneven_groups()
    cands = synth.make_candidates(sum(counts), seed=4)
    with k2.Plan(t, counts, ks, Ts, tol=TOL) as plan:
        val, dd, dk = plan.run(cands)
        off = 0
        for g, (c, k, T) in enumerate(zip(counts, ks, Ts)):
            idx = off + np.unique(np.array([0, c // 3, (2 * c) // 3, c - 1]))
            assert len(idx) == 4
            n_T = t.count_below(T)
            ohi, _ = oracle.k2(cands.subset(idx), data, k, n_T)
            gi = _check_bounds(plan, g, np.stack([val[idx], dd[idx], dk[idx]]), ohi)
            assert gi["n_T"] == n_T and gi["err_bound"] <= TOL
            off += c
        # the same bits under the one-kernel schedules, twelve uneven groups in one launch
        for sched in (1, 2, 3):
            plan.set_schedule(sched)
            for x, y in zip(plan.run(cands), (val, dd, dk)):
                assert np.array_equal(x, y), sched


def test_newton_polish_derivatives_vs_oracle(big, oracle):
    import torch
    from mertens_bound_b200.autograd import K2Torch
    data, t = big
    K, T = 1.5e-10, 1.3e6
    cands = synth.make_candidates(1024, seed=5)
    cands.delta[:] = np.random.default_rng(55).uniform(-5e-5, 5e-5, 1024)
    dev = torch.device("cuda", 0)
    vi = torch.from_numpy(cands.v_int.view(np.int64).copy()).to(dev)
    vf = torch.from_numpy(cands.v_frac.view(np.int64).copy()).to(dev)
    d = torch.from_numpy(cands.delta.copy()).to(dev)
    n_T = t.count_below(T)
    assert n_T == 2_325_572
    ev = K2Torch(t, T=T, tol=TOL)
    try:
        plan = ev.plan(1024, K)
        # value and both derivatives through the autograd wrapper
        dg = d.clone().requires_grad_(True)
        kk = torch.tensor(K, dtype=torch.float64, device=dev, requires_grad=True)
        val = ev(vi, vf, dg, kk)
        val.sum().backward()
        sel = np.arange(0, 1024, 64)                       # 16 candidates
        ohi, _ = oracle.k2(cands.subset(sel), data, K, n_T)
        got = np.stack([val.detach().cpu().numpy()[sel], dg.grad.cpu().numpy()[sel],
                        np.full(len(sel), np.nan)])
        _, dd, dk = ev.evaluate(vi, vf, d, K)
        got[2] = dk.cpu().numpy()[sel]
        _check_bounds(plan, 0, got, ohi)
        # the certified enclosures of K2 and both derivatives at the same 16 points (delta folded
        # into the 64.64 base, rounded to nearest 2^-64 as the plan does; v_rad covers the rounding):
        # each autograd output lies within its a-priori bound of its interval
        from fractions import Fraction
        pts = []
        for i in sel:
            x = (int(cands.v_int[i]) << 64) + int(cands.v_frac[i]) + Fraction(float(cands.delta[i])) * 2 ** 64
            pts.append(int(x + Fraction(1, 2)) if x >= 0 else int(x - Fraction(1, 2)))
        cb = synth.Candidates(np.array([x >> 64 for x in pts], np.uint64),
                              np.array([x & ((1 << 64) - 1) for x in pts], np.uint64), np.zeros(len(sel)))
        clo, chi = k2.k2_certified_grad(t, cb, K, T, v_rad=2.0 ** -64)
        gi = plan.group_info(0)
        for q, key in ((0, "err_bound"), (1, "err_bound_dd"), (2, "err_bound_dk")):
            dist = np.maximum(np.maximum(clo[q] - got[q], got[q] - chi[q]), 0.0)
            assert np.max(dist) <= gi[key], (key, np.max(dist), gi[key])
            ulp = np.spacing(np.abs(ohi[:, q]))               # the oracle's value rounded to FP64
            assert np.all(clo[q] - ulp <= ohi[:, q]) and np.all(ohi[:, q] <= chi[q] + ulp), key
        # k.grad = sum_p dK2_p/dk
        gk = float(kk.grad.item())
        assert abs(gk - float(dk.sum().item())) <= 1e-12 * float(dk.abs().sum().item())
        # central differences at delta step 1e-4 against the oracle's own difference quotient
        h = 1e-4
        fsel = sel[:8]
        vp, _, _ = ev.evaluate(vi, vf, d + h, K)
        vm, _, _ = ev.evaluate(vi, vf, d - h, K)
        fd = ((vp - vm) / (2 * h)).cpu().numpy()[fsel]
        cp, cm = cands.subset(fsel), cands.subset(fsel)
        cp.delta[:] = cands.delta[fsel] + h
        cm.delta[:] = cands.delta[fsel] - h
        op, _ = oracle.k2(cp, data, K, n_T)
        om, _ = oracle.k2(cm, data, K, n_T)
        ofd = (op[:, 0] - om[:, 0]) / (2 * h)
        eb = plan.group_info(0)["err_bound"]
        assert np.max(np.abs(fd - ofd)) <= 2 * eb / (2 * h) + 1e-9
        # 8 batched Newton steps on delta: |K2| never decreases, the slope vanishes where it moved
        dn = d.clone()
        h0, v8, d8, k8 = ev.newton(vi, vf, dn, K, iters=8, max_step=1e-4)
        h0, v8 = h0.cpu().numpy(), v8.cpu().numpy()
        assert np.all(np.abs(v8) >= np.abs(h0))
        moved = dn.cpu().numpy() != cands.delta
        assert moved.sum() >= 512
        nsel = np.flatnonzero(moved)[:4]
        cn = cands.subset(nsel)
        cn.delta[:] = dn.cpu().numpy()[nsel]
        on, _ = oracle.k2(cn, data, K, n_T)
        assert np.max(np.abs(v8[nsel] - on[:, 0])) <= eb
    finally:
        ev.close()
