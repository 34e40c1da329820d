"""The per-peak polish contracts of search/path1_kernel_opt.py on the GPU against the reference's
own outputs (tests/golden/path1_polish.json), the oracle, and the fused (matrix-free) forms."""
import json
import os

import numpy as np
import pytest

from mertens_bound_b200 import k2, path1, synth

pytestmark = pytest.mark.gpu

FX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "path1_polish.json")


@pytest.fixture(scope="module")
def fx():
    return json.load(open(FX))


@pytest.fixture(scope="module")
def setup(gpu, fx, oracle):
    t = synth.make_table(fx["table"]["n"], seed=fx["table"]["seed"])
    c = synth.make_candidates(fx["candidates"]["P"], seed=fx["candidates"]["seed"])
    n = fx["n_zeros"]
    A, B = oracle.exact_AB(c, t, n)
    table = k2.ZeroTable.from_data(t)
    yield t, c, n, A, B, table
    table.close()


def weights(gamma):
    u = gamma / gamma[-1]
    return {"jp": (1.0 - u) * np.cos(np.pi * u) + np.sin(np.pi * u) / np.pi,
            "g3e-9": np.exp(-3e-9 * gamma * gamma)}


def test_exact_AB_vs_oracle(setup, oracle):
    t, c, n, A, B, table = setup
    gA, gB = path1.compute_exact_AB(table, c, n)
    scale = 2 * np.hypot(t.c_re[:n], t.c_im[:n])
    assert np.max(np.abs(gA - A) / scale) <= 4e-16
    assert np.max(np.abs(gB - B) / scale) <= 4e-16
    # with an FP64 offset: angle error below 2 pi |delta| 2^-52
    cd = c.subset(np.arange(16))
    cd.delta[:] = np.random.default_rng(4).uniform(-1e-4, 1e-4, 16)
    gA, gB = path1.compute_exact_AB(table, cd, n)
    qA, qB = oracle.exact_AB(cd, t, n)
    assert np.max(np.abs(gA - qA) / scale) <= 6e-16
    assert np.max(np.abs(gB - qB) / scale) <= 6e-16


@pytest.mark.parametrize("name", ["jp", "g3e-9"])
def test_polish_single_vs_reference(setup, fx, name):
    t, c, n, A, B, _ = setup
    g = t.gamma[:n]
    w = weights(g)[name]
    hu, hp, dp = path1.polish_single_peak(A[:8], B[:8], g, w, n_zeros=n, grid_hw=4e-5, grid_steps=40)
    want = np.array(fx[name]["single_first8"])
    np.testing.assert_allclose(hu, want[:, 0], rtol=1e-11, atol=1e-14)
    np.testing.assert_allclose(hp, want[:, 1], rtol=1e-11, atol=1e-14)
    np.testing.assert_allclose(dp, want[:, 2], rtol=0, atol=1e-12)
    # one peak, 1-D form
    h0, h1, d1 = path1.polish_single_peak(A[3], B[3], g, w, n_zeros=n)
    assert (h0, h1, d1) == (hu[3], hp[3], dp[3])


@pytest.mark.parametrize("name", ["jp", "g3e-9"])
def test_fast_polish_vs_reference(setup, fx, name):
    t, c, n, A, B, _ = setup
    g = t.gamma[:n]
    hu, hp, dp = path1.fast_polish_batch(A, B, g, weights(g)[name])
    want = fx[name]["batch"]
    np.testing.assert_allclose(hu, want["h_unpol"], rtol=1e-11, atol=1e-14)
    np.testing.assert_allclose(hp, want["h_pol"], rtol=1e-11, atol=1e-14)
    np.testing.assert_allclose(dp, want["ddy_pol"], rtol=0, atol=1e-12)


def test_fused_forms_match_matrix_forms(setup):
    """(A, B) computed on the fly give the matrix forms' results on the exact A/B."""
    t, c, n, _, _, table = setup
    gA, gB = path1.compute_exact_AB(table, c, n)
    w = np.zeros(t.n)
    w[:n] = weights(t.gamma[:n])["jp"]
    slot = table.add_weights(w)
    g = t.gamma[:n]
    mu, mp, md = path1.polish_single_peak(gA[:8], gB[:8], g, w[:n], n_zeros=n)
    eu, ep, ed = path1.polish_single_exact(table, c.subset(np.arange(8)), slot, n)
    np.testing.assert_allclose(eu, mu, rtol=1e-13, atol=1e-16)
    np.testing.assert_allclose(ep, mp, rtol=1e-13, atol=1e-16)
    np.testing.assert_allclose(ed, md, rtol=0, atol=1e-14)
    mu, mp, md = path1.fast_polish_batch(gA, gB, g, w[:n], top=10)
    eu, ep, ed = path1.fast_polish_exact(table, c, slot, n, top=10)
    np.testing.assert_allclose(eu, mu, rtol=1e-13, atol=1e-16)
    np.testing.assert_allclose(ep, mp, rtol=1e-13, atol=1e-16)
    np.testing.assert_allclose(ed, md, rtol=0, atol=1e-14)


def test_edge_cases(setup):
    t, c, n, A, B, table = setup
    g = t.gamma[:n]
    w = weights(g)["jp"]
    # no grid: Newton from 0 only
    hu, hp, dp = path1.polish_single_peak(A[:4], B[:4], g, w, n_zeros=n, grid_steps=0)
    assert np.all(np.abs(hp) >= np.abs(hu))
    # top = 0: the Taylor grid values only; one grid point
    hu, hp, dp = path1.fast_polish_batch(A[:5], B[:5], g, w, ddy_grid=np.array([0.0]), top=0)
    np.testing.assert_allclose(hp, hu, rtol=1e-15, atol=0)
    assert np.all(dp == 0.0)
    # empty batch, zero zeros
    e = path1.fast_polish_batch(np.zeros((0, n)), np.zeros((0, n)), g, w)
    assert all(x.shape == (0,) for x in e)
    hu, hp, dp = path1.polish_single_peak(A[:2, :0], B[:2, :0], g[:0], w[:0])
    assert np.all(hu == 0) and np.all(hp == 0) and np.all(dp == 0)
    # argument errors
    from mertens_bound_b200._lib import K2Error
    with pytest.raises(K2Error, match="MB_ERR_ARG"):
        path1.fast_polish_exact(table, c, 99, n)
    with pytest.raises(K2Error, match="MB_ERR_ARG"):
        path1.fast_polish_batch(A[:2], B[:2], g, w, ddy_grid=np.array([np.nan]))
    bad = c.subset(np.arange(2))
    bad.delta[:] = [0.0, 1e6]
    with pytest.raises(K2Error, match="MB_ERR_ARG"):
        path1.compute_exact_AB(table, bad, 10)
