"""Golden fixtures (tests/golden/, made by make_golden.py): the oracle pinned to the reference's
own evaluator outputs and to the interval balls, and the GPU kernels checked against them."""
import json
import math
import os
from fractions import Fraction

import numpy as np
import pytest

from mertens_bound_b200 import k2, synth

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    p = os.path.join(HERE, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} not generated")
    return json.load(open(p))


def _sha(t):
    import hashlib
    h = hashlib.sha256()
    for a in (t.G3, t.gamma, t.c_re, t.c_im):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _cands(fx):
    return synth.Candidates(np.array([int(x) for x in fx["v_int"]], np.uint64),
                            np.array([int(x) for x in fx["v_frac"]], np.uint64), np.zeros(len(fx["v_int"])))


@pytest.fixture(scope="module")
def small():
    fx = _load("small_plain.json")
    t = synth.make_table(fx["table"]["n"], seed=fx["table"]["seed"])
    assert _sha(t) == fx["table"]["sha256"], "synthetic generator changed; regenerate the fixtures"
    return fx, t, _cands(fx)


def test_oracle_reproduces_fixture(small, oracle):
    fx, t, c = small
    hi, lo = oracle.k2(c, t, fx["k"], t.n)
    for q, key in enumerate(("val", "dd", "dk")):
        want = np.array(fx["oracle_k2"][key])
        assert np.array_equal(hi[:, q], want[:, 0])


def test_oracle_pinned_to_reference_evaluator_outputs(small, oracle):
    """h0 from the reference's compiled compute_peak_AB + polish_peaks_with_weights
    (recorded in the fixture) agrees with the binary128 oracle to FP64 rounding."""
    fx, t, c = small
    if "reference_evaluator" not in fx:
        pytest.skip("fixture made without the reference evaluator")
    h0 = np.array(fx["reference_evaluator"]["h0"])
    want = np.array(fx["oracle_k2"]["val"])[:, 0]
    assert np.max(np.abs(h0 - want)) < 5e-14


# the binary128 oracle's own accumulated rounding (113-bit terms, up to 2.3e6 of them) is far
# below the 1e-10 bar but above the 220-bit balls' width: compare with this slack
QUAD_SLACK = Fraction(1, 10 ** 26)


def test_interval_balls_contain_oracle(small):
    fx, t, c = small
    for p, (a, b) in enumerate(fx["interval_balls_first4"]):
        hi, lo = fx["oracle_k2"]["val"][p]
        x = Fraction(hi) + Fraction(lo)
        assert Fraction(a) - QUAD_SLACK <= x <= Fraction(b) + QUAD_SLACK
        assert Fraction(b) - Fraction(a) < Fraction(1, 10 ** 30)


def test_derivative_balls_contain_oracle(small):
    """dK2/ddelta and dK2/dk of the binary128 oracle inside the 220-bit interval derivatives."""
    fx, t, c = small
    if "derivative_balls_first4" not in fx:
        pytest.skip("fixture made without derivative balls")
    for p, balls in enumerate(fx["derivative_balls_first4"]):
        for key in ("dd", "dk"):
            a, b = (Fraction(x) for x in balls[key])
            hi, lo = fx["oracle_k2"][key][p]
            x = Fraction(hi) + Fraction(lo)
            slack = abs(x) * Fraction(1, 10 ** 28)
            assert a - slack <= x <= b + slack, (p, key)
            assert b - a <= abs(x) * Fraction(1, 10 ** 40)


def test_exact_phases(small, oracle):
    fx, t, c = small
    for e in fx["exact_phases"]:
        hi, lo = oracle.phase128(c.subset(np.array([e["p"]])), t.G3[e["j"]:e["j"] + 1])
        assert (int(hi[0, 0]), int(lo[0, 0])) == (int(e["hi"]), int(e["lo"]))


def test_full_ball_contains_oracle():
    fx = _load("peak2_full_ball.json")
    x = Fraction(fx["oracle_k2"][0]) + Fraction(fx["oracle_k2"][1])
    assert Fraction(fx["ball_lo"]) - QUAD_SLACK <= x <= Fraction(fx["ball_hi"]) + QUAD_SLACK
    assert fx["ball_width"] < 1e-40


# ------------------------------------------------------------------ GPU kernels vs fixtures

@pytest.mark.gpu
def test_kernels_against_fixture(gpu, small):
    fx, t, c = small
    with k2.ZeroTable.from_data(t) as tb:
        phi, _ = k2.phase128(tb, c, t.n)
        for e in fx["exact_phases"]:
            assert int(phi[e["p"], e["j"]]) == int(e["hi"])
        val, dd, dk = k2.k2_plain(tb, c, fx["k"])
        want = np.array(fx["oracle_k2"]["val"])[:, 0]
        assert np.max(np.abs(val - want)) < 2e-13
        fv, fd, fk, eb = k2.k2_fast(tb, c, fx["k"])
        assert np.max(np.abs(fv - want)) <= eb <= 1e-10
        # derivatives against the 220-bit interval derivatives (the "Arb derivative")
        for p, balls in enumerate(fx.get("derivative_balls_first4", [])):
            for key, plain_v, fast_v in (("dd", dd[p], fd[p]), ("dk", dk[p], fk[p])):
                a, b = (float(Fraction(x)) for x in balls[key])
                mid = 0.5 * (a + b)
                assert abs(plain_v - mid) <= 1e-10 * abs(mid), (p, key)
                assert abs(fast_v - mid) <= 1e-6 * abs(mid), (p, key)
        lo, hi, _ = k2.k2_certified(tb, c.subset(np.arange(4)), fx["k"])
        for p, (a, b) in enumerate(fx["interval_balls_first4"]):
            assert Fraction(lo[p]) <= Fraction(a) and Fraction(b) <= Fraction(hi[p])


@pytest.mark.gpu
def test_certified_full_sum_contains_ball(gpu):
    """The directed-rounding interval over all 2,325,572 zeros at Peak2 contains the committed
    interval ball computed from the same stored gamma_j (G_j) and c_j."""
    fx = _load("peak2_full_ball.json")
    t = synth.make_table(fx["table"]["n"], seed=fx["table"]["seed"])
    assert _sha(t) == fx["table"]["sha256"]
    c = synth.Candidates(np.array([int(fx["v_int"])], np.uint64), np.array([int(fx["v_frac"])], np.uint64),
                         np.zeros(1))
    with k2.ZeroTable.from_data(t) as tb:
        lo, hi, _ = k2.k2_certified(tb, c, fx["k"], fx["T0"])
    assert Fraction(lo[0]) <= Fraction(fx["ball_lo"]) and Fraction(fx["ball_hi"]) <= Fraction(hi[0])
    assert hi[0] - lo[0] < 1e-11
