"""Plans scored under per-zero weight vectors (the search drivers' JP, raw and cutoff kernels,
search/eval_tech1_600k.py:243-249) against the oracle's weighted binary128 sum."""
import math

import numpy as np
import pytest

from mertens_bound_b200 import k2, synth
from mertens_bound_b200._lib import K2Error

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.fixture(scope="module")
def table(gpu, small_table):
    t = k2.ZeroTable.from_data(small_table)
    yield t
    t.close()


def weight_vectors(gamma):
    u = gamma / gamma[-1]
    jp = (1.0 - u) * np.cos(np.pi * u) + np.sin(np.pi * u) / np.pi
    raw = np.ones_like(gamma)
    cut = np.zeros_like(gamma)
    cut[:5000] = 1.0
    g15 = np.exp(-1.5e-10 * gamma * gamma)
    return {"jp": jp, "raw": raw, "cut5k": cut, "g15": g15}


def test_weighted_groups_vs_oracle(table, small_table, oracle):
    W = weight_vectors(small_table.gamma)
    names = list(W)
    slots = [table.add_weights(W[n]) for n in names]
    per = 48
    counts = [per] * (len(names) + 1)
    ks = [0.0] * len(names) + [3e-9]
    Ts = [math.inf] * (len(names) + 1)
    cd = synth.make_candidates(per * len(counts), seed=41)
    with k2.Plan(table, counts, ks, Ts, tol=TOL, weights=slots + [-1]) as plan:
        val, dd, dk = plan.run(cd)
        for g, name in enumerate(names + ["gauss"]):
            sub = cd.subset(np.arange(g * per, (g + 1) * per))
            w = W[name] if name != "gauss" else None
            ohi, _ = oracle.k2(sub, small_table, ks[g], small_table.n, weights=w)
            eb = plan.group_info(g)["err_bound"]
            assert eb <= TOL
            sl = slice(g * per, (g + 1) * per)
            assert np.max(np.abs(val[sl] - ohi[:, 0])) <= eb, name
            assert np.max(np.abs(dd[sl] - ohi[:, 1])) <= 1e-6 * np.max(np.abs(ohi[:, 1])), name
            assert np.max(np.abs(dk[sl] - ohi[:, 2])) <= 1e-6 * np.max(np.abs(ohi[:, 2])), name


def test_gaussian_weight_vector_matches_k(table, small_table):
    """A weight vector equal to exp(-k gamma^2) gives the Gaussian group's values."""
    k = 1.5e-10
    slot = table.add_weights(np.exp(-k * small_table.gamma * small_table.gamma))
    cd = synth.make_candidates(256, seed=42)
    cd.delta[:] = np.random.default_rng(5).uniform(-1e-4, 1e-4, 256)
    with k2.Plan(table, [256], [k], [30000.0], tol=TOL, weights=[slot]) as pw, \
            k2.Plan(table, [256], [k], [30000.0], tol=TOL) as pg:
        vw, dw, _ = pw.run(cd)
        vg, dg, _ = pg.run(cd)
        eb = pw.group_info(0)["err_bound"] + pg.group_info(0)["err_bound"]
        assert np.max(np.abs(vw - vg)) <= eb
        assert np.max(np.abs(dw - dg)) <= 1e-6 * np.max(np.abs(dg))


def test_weight_errors(table, small_table):
    with pytest.raises(ValueError):
        table.add_weights(np.ones(small_table.n - 1))
    bad = np.ones(small_table.n)
    bad[17] = np.nan
    with pytest.raises(K2Error, match="MB_ERR_TABLE"):
        table.add_weights(bad)
    with pytest.raises(K2Error, match="MB_ERR_ARG"):
        k2.Plan(table, [4], [0.0], [math.inf], weights=[63])
    with pytest.raises(ValueError):
        k2.Plan(table, [4, 4], [0.0, 0.0], [math.inf, math.inf], weights=[-1])
