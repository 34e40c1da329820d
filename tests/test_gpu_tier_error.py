"""The per-term error model behind the a-priori bounds, tested term by term: one-zero tables
(a low and a high zero), 2^18 random candidates, every term evaluated in the light tier (tol
large) or in the heavy tier (tol tiny), each K2 = a cos(theta + arg c) checked against the
binary128 oracle within its plan's bound (EPS_LIGHT a or EPS_HEAVY a, plus FP64 roundings)."""
import math

import numpy as np
import pytest

from mertens_bound_b200 import k2, synth

pytestmark = pytest.mark.gpu

P = 1 << 18


def one_zero(j):
    """Zero j of the synthetic table, or (j a float) one zero at gamma = j with random low bits of G
    and the coefficient of the table's last zero below 3e5."""
    if isinstance(j, float):
        t = synth.make_table_below(3e5, seed=1)
        G3 = synth.fixed_from_double(np.array([j / (2.0 * math.pi)]), np.random.default_rng(11))
        return synth.ZeroTableData(G3, synth.gamma_from_fixed(G3), t.c_re[-1:].copy(), t.c_im[-1:].copy(), t.seed)
    t = synth.make_table_below(3e5, seed=1) if j > 0 else synth.make_table(1, seed=5)
    return synth.ZeroTableData(t.G3[j:j + 1].copy(), t.gamma[j:j + 1].copy(), t.c_re[j:j + 1].copy(),
                               t.c_im[j:j + 1].copy(), t.seed)


# 3.2e6: the light tier's one-FMA fraction product at an integer part of G near its 2^19 limit;
# 5e6: above the limit, the split light phase
@pytest.mark.parametrize("j", [0, 400_000, 3.2e6, 5.0e6])
@pytest.mark.parametrize("tier,tol", [("light", 1.0), ("heavy", 1e-30)])
def test_per_term_error_within_bound(gpu, oracle, j, tier, tol):
    data = one_zero(j)
    cd = synth.make_candidates(P, seed=17 + int(j))
    ohi, _ = oracle.k2(cd, data, 0.0, 1)
    with k2.ZeroTable.from_data(data) as t, k2.Plan(t, [P], [0.0], [math.inf], tol=tol) as plan:
        gi = plan.group_info(0)
        assert gi["n_heavy"] == (0 if tier == "light" else 1)
        val, dd, dk = plan.run(cd)
    a = 2 * math.hypot(data.c_re[0], data.c_im[0])
    err = np.abs(val - ohi[:, 0])
    assert np.max(err) <= gi["err_bound"], (tier, np.max(err) / a)
    assert np.max(np.abs(dd - ohi[:, 1])) <= gi["err_bound_dd"]
    assert np.max(np.abs(dk - ohi[:, 2])) <= gi["err_bound_dk"]
    # the light bound is not vacuous: the worst observed error is within 100x of it
    assert np.max(err) >= gi["err_bound"] / 100 or tier == "heavy"
