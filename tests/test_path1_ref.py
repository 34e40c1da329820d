"""The oracle's restatements of search/path1_kernel_opt.py pinned to the reference's own outputs
(tests/golden/path1_polish.json, made by tests/golden/make_golden.py)."""
import hashlib
import json
import os

import numpy as np
import pytest

from mertens_bound_b200 import synth

FX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "path1_polish.json")


@pytest.fixture(scope="module")
def fx():
    return json.load(open(FX))


@pytest.fixture(scope="module")
def inputs(fx, oracle):
    t = synth.make_table(fx["table"]["n"], seed=fx["table"]["seed"])
    c = synth.make_candidates(fx["candidates"]["P"], seed=fx["candidates"]["seed"])
    n = fx["n_zeros"]
    A, B = oracle.exact_AB(c, t, n)
    return t, c, n, A, B


def weights(gamma):
    u = gamma / gamma[-1]
    return {"jp": (1.0 - u) * np.cos(np.pi * u) + np.sin(np.pi * u) / np.pi,
            "g3e-9": np.exp(-3e-9 * gamma * gamma)}


def test_oracle_AB_reproduces_fixture_inputs(fx, inputs):
    _, _, _, A, B = inputs
    assert hashlib.sha256(A.tobytes() + B.tobytes()).hexdigest() == fx["AB_sha256"]


def test_oracle_AB_matches_256bit(fx, inputs):
    """binary128 A/B rounded to FP64 equal the 256-bit values rounded to FP64 (to 1 ulp)."""
    _, _, _, A, B = inputs
    for q in fx["exact_AB_pairs_256bit"]:
        for got, want in ((A[q["p"], q["j"]], q["A"]), (B[q["p"], q["j"]], q["B"])):
            assert abs(got - want) <= np.spacing(abs(want)), (q, got, want)


@pytest.mark.parametrize("name", ["jp", "g3e-9"])
def test_polish_single_restatement(fx, inputs, name):
    from oracle import polish_ref
    t, _, n, A, B = inputs
    g = t.gamma[:n]
    w = weights(g)[name]
    for p, want in enumerate(fx[name]["single_first8"]):
        got = polish_ref.polish_single_peak(A[p], B[p], g, w, n_zeros=n, grid_hw=4e-5, grid_steps=40)
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("name", ["jp", "g3e-9"])
def test_fast_polish_restatement(fx, inputs, name):
    from oracle import polish_ref
    t, _, n, A, B = inputs
    g = t.gamma[:n]
    hu, hp, dp = polish_ref.fast_polish_batch(A, B, g, weights(g)[name])
    want = fx[name]["batch"]
    np.testing.assert_allclose(hu, want["h_unpol"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(hp, want["h_pol"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(dp, want["ddy_pol"], rtol=1e-12, atol=1e-15)
