"""Plain FP64 kernel and exact phase on the GPU, against the oracle."""
import math

import numpy as np
import pytest

from mertens_bound_b200 import k2, synth

pytestmark = pytest.mark.gpu

MASK64 = (1 << 64) - 1


@pytest.fixture(scope="module")
def table(gpu, small_table):
    t = k2.ZeroTable.from_data(small_table)
    yield t
    t.close()


def test_phase_bit_exact(table, small_table, oracle):
    cd = synth.make_candidates(64, seed=21)
    hi, lo = k2.phase128(table, cd, 2000)
    ohi, olo = oracle.phase128(cd, small_table.G3, 2000)
    assert np.array_equal(hi, ohi) and np.array_equal(lo, olo)


def test_phase_edge_candidates(table, small_table, oracle):
    cd = synth.Candidates(np.array([MASK64, 0, 1, 3_484_971_332_733_132_396], dtype=np.uint64),
                          np.array([MASK64, 0, MASK64, 9_930_597_040_327_004_160], dtype=np.uint64), np.zeros(4))
    hi, lo = k2.phase128(table, cd, 1000)
    ohi, olo = oracle.phase128(cd, small_table.G3, 1000)
    assert np.array_equal(hi, ohi) and np.array_equal(lo, olo)


@pytest.mark.parametrize("P", [1, 5, 64, 300])
def test_plain_vs_oracle(table, small_table, oracle, P):
    cd = synth.make_candidates(P, seed=30 + P)
    k = 3e-9
    val, dd, dk = k2.k2_plain(table, cd, k)
    ohi, olo = oracle.k2(cd, small_table, k, small_table.n)
    # tolerance: FP64 term errors ~1e-16 * sum|term| (sum ~ 4) plus summation
    assert np.max(np.abs(val - ohi[:, 0])) < 2e-13
    assert np.max(np.abs(dd - ohi[:, 1])) < 2e-13 * np.max(np.abs(ohi[:, 1]))
    assert np.max(np.abs(dk - ohi[:, 2])) < 2e-13 * np.max(np.abs(ohi[:, 2]))


def test_plain_cutoff_and_delta(table, small_table, oracle):
    cd = synth.make_candidates(32, seed=41)
    cd.delta[:] = np.linspace(-3e-4, 3e-4, 32)
    k, T = 1e-9, 5000.0
    n_use = small_table.count_below(T)
    assert table.count_below(T) == n_use
    val, dd, dk = k2.k2_plain(table, cd, k, T)
    ohi, _ = oracle.k2(cd, small_table, k, n_use)
    assert np.max(np.abs(val - ohi[:, 0])) < 2e-13
    assert np.max(np.abs(dd - ohi[:, 1])) < 2e-13 * np.max(np.abs(ohi[:, 1]))


def test_plain_empty_cutoff(table):
    cd = synth.make_candidates(3, seed=1)
    val, dd, dk = k2.k2_plain(table, cd, 3e-9, T=1.0)
    assert np.all(val == 0) and np.all(dd == 0) and np.all(dk == 0)
