"""The oracle itself: exact phase against Python integers, binary128 sums against the
reference's own compiled evaluator (oracle/_ref), and against the committed golden vectors."""
import numpy as np
import pytest

from mertens_bound_b200 import synth
from oracle.oracle import RefLib, phase128_bigint, reference_candidates, reference_format

MASK64 = (1 << 64) - 1


def test_phase_c_matches_bigint(oracle, small_table):
    cd = synth.make_candidates(6, seed=11)
    # edge candidates: all-ones limbs, zero fraction, maximal integer part
    extra = synth.Candidates(np.array([MASK64, 0, 3_600_000_000_000_000_000], dtype=np.uint64),
                             np.array([MASK64, 0, 1], dtype=np.uint64), np.zeros(3))
    for c in (cd, extra):
        hi, lo = oracle.phase128(c, small_table.G3[:300])
        for p in range(c.n):
            for j in range(0, 300, 7):
                h, l = phase128_bigint(c.v_int[p], c.v_frac[p], small_table.G3[j])
                assert (int(hi[p, j]), int(lo[p, j])) == (h, l)


def test_phase_edge_limbs(oracle):
    G3 = np.array([[0, 0, 0], [0xFFFFFFFF, MASK64, MASK64], [1, 1 << 63, 1], [123456, MASK64, 0]], dtype=np.uint64)
    c = synth.Candidates(np.array([MASK64, 1, 0], dtype=np.uint64), np.array([MASK64, MASK64, 1], dtype=np.uint64), np.zeros(3))
    hi, lo = oracle.phase128(c, G3)
    for p in range(3):
        for j in range(4):
            assert (int(hi[p, j]), int(lo[p, j])) == phase128_bigint(c.v_int[p], c.v_frac[p], G3[j])


def test_interval_ball_contains_quad(oracle, small_table):
    """The mpmath interval restatement of the Arb sum encloses the binary128 value and is
    far narrower than the 1e-10 bar."""
    from fractions import Fraction
    from oracle.interval import bounds, k2_ball
    n = 300
    cd = synth.make_candidates(2, seed=14)
    cd.delta[:] = [0.0, 3e-5]
    hi, lo = oracle.k2(cd, small_table, 3e-9, n)
    for p in range(2):
        val, dd, dk = k2_ball(cd.v_int[p], cd.v_frac[p], cd.delta[p], small_table.G3, small_table.c_re,
                              small_table.c_im, 3e-9, n)
        for q, ball in enumerate((val, dd, dk)):
            a, b = bounds(ball)
            x = Fraction(float(hi[p, q])) + Fraction(float(lo[p, q]))
            width = max(abs(float(b)), 1.0) * 1e-25
            assert a - Fraction(width) <= x <= b + Fraction(width)
            assert float(b - a) < 1e-30 * max(1.0, abs(float(a)))


@pytest.mark.skipif(not RefLib.available(), reason="reference evaluator not built")
def test_quad_oracle_matches_reference_evaluator(oracle, small_table):
    """K2 from the reference's compute_peak_AB + h0 (path1_eval_fast.cpp:15-53, :76-81) on the
    same table in the reference layout agrees with the binary128 oracle to FP64 rounding."""
    t = small_table.truncate(3000)
    cd = synth.make_candidates(16, seed=12)
    k = 3e-9
    hi, _ = oracle.k2(cd, t, k, t.n)
    R = RefLib()
    A, B = R.peak_AB(reference_candidates(cd), reference_format(t))
    w = np.exp(-k * t.gamma ** 2)
    h0, _, _ = R.polish(A, B, t.gamma, w, 2.5e-4, 0)
    assert np.max(np.abs(h0 - hi[:, 0])) < 5e-14
    dd = -(B @ (w * t.gamma))
    dk = -(A @ (w * t.gamma ** 2))
    assert np.max(np.abs(dd - hi[:, 1])) < 1e-14 * np.max(np.abs(hi[:, 1])) * 100
    assert np.max(np.abs(dk - hi[:, 2])) < 1e-14 * np.max(np.abs(hi[:, 2])) * 100


@pytest.mark.skipif(not RefLib.available(), reason="reference evaluator not built")
def test_reference_phase_reduction_restated(oracle, small_table):
    """path1_eval_fast.cpp:45-46 with dy0 = 0 (fraction bits below 2^-34 zero) gives the exact
    phase plus arg(c)/2pi in its top word, to within one unit of 2^-64."""
    t = small_table.truncate(500)
    cd = synth.make_candidates(4, seed=13)
    cd.v_frac[:] = cd.v_frac & ~np.uint64((1 << 34) - 1)
    reft = reference_format(t)
    A, B, top = oracle.ref_peak_AB(reference_candidates(cd), reft, want_top=True)
    hi, lo = oracle.phase128(cd, t.G3)
    for p in range(cd.n):
        for j in range(t.n):
            psi = (int(reft["psi_hi"][j]) << 64) | int(reft["psi_lo"][j])
            want = ((((int(hi[p, j]) << 64) | int(lo[p, j])) - psi) % (1 << 128)) >> 64
            d = (int(top[p, j]) - want) % (1 << 64)
            assert d in (0, 1, (1 << 64) - 1)


def test_fast_screen_restatement(oracle):
    """The C restatement of ZeroData::fast_screen (search/fast_mertens_enum.cpp:99-142) against a
    pure-Python one: u128 phase, 14-bit index into the FP32 cosine table, seven offsets, FP32
    sums in the reference's order, stage thresholds 0.810 / 0.875.  The amplitudes are scaled up
    so that leaves pass, fail at the first stage and fail at the second."""
    import math
    d = synth.make_table(2000, seed=3)
    reft = reference_format(d, exact_psi=False)
    ta = 4.0 * 2.0 * reft["alpha"] * np.exp(-3e-9 * d.gamma ** 2)
    rng = np.random.default_rng(1)
    xs = [int(rng.integers(3_400_000_000_000_000_000, 3_600_000_000_000_000_000)) << 30 |
          int(rng.integers(0, 1 << 30)) for _ in range(160)]
    flags = oracle.fast_screen(np.array([x & MASK64 for x in xs], np.uint64),
                               np.array([x >> 64 for x in xs], np.uint64), reft, ta)
    f32 = np.float32
    lut = np.array([math.cos(2.0 * math.pi * k / 16384.0) for k in range(16384)]).astype(np.float32)
    st = [int(round(g * 0.0014 * (16384.0 / (2.0 * math.pi)))) & 16383 for g in d.gamma[:128]]
    limbs = [((int(reft["ghi_hi"][i]) << 64) | int(reft["ghi_lo"][i]),
              (int(reft["glo_hi"][i]) << 64) | int(reft["glo_lo"][i]),
              (int(reft["psi_hi"][i]) << 64) | int(reft["psi_lo"][i])) for i in range(128)]

    def screen(x):
        xh, xl = x >> 48, x & ((1 << 48) - 1)
        s = [f32(0)] * 7
        for stage, thr in ((0, f32(0.810)), (1, f32(0.875))):
            for i in range(64 * stage, 64 * stage + 64):
                ghi, glo, psi = limbs[i]
                i0 = ((xh * ghi + xl * glo - psi) % (1 << 128)) >> 114
                w = f32(ta[i])
                for m in range(7):
                    s[m] = f32(s[m] + f32(w * lut[(i0 + (m - 3) * st[i]) % 16384]))
            if max(abs(v) for v in s) < thr:
                return 0, stage
        return 1, 2

    res = [screen(x) for x in xs]
    assert [r[0] for r in res] == flags.tolist()
    outcomes = {r[1] for r in res}
    assert outcomes == {0, 1, 2}, outcomes
