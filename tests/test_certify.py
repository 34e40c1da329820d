"""certify_K2 contract: exact enclosures of decimal inputs and ball strings (CPU), and the GPU
certificate (one-shot and batched with the key-checked cache) against the oracle."""
import json
import math
import os
from fractions import Fraction

import numpy as np
import pytest

from mertens_bound_b200 import certify, synth


# ------------------------------------------------------------------ CPU: exact helpers

def test_k_interval_encloses_decimal():
    lo, hi = certify.k_interval("1.5e-10")
    q = Fraction("1.5e-10")
    assert Fraction(lo) <= q <= Fraction(hi) and lo < hi
    assert certify.k_interval("0.5") == (0.5, 0.5)


def test_v_point_encloses_decimal():
    vi, vf, rad = certify.v_point(synth.PEAK2_STR)
    q = Fraction(synth.PEAK2_STR)
    base = Fraction(vi) + Fraction(vf, 1 << 64)
    assert base <= q <= base + Fraction(rad) and rad < 2.0 ** -64


@pytest.mark.parametrize("lo,hi", [(1.0003052504, 1.0003052505), (-2.5e-7, -2.4e-7), (0.0, 3e-12), (5, 5)])
def test_ball_encloses(lo, hi):
    s = certify.ball(lo, hi, 15)
    a, b = certify.ball_bounds(s)
    assert a <= Fraction(lo) and Fraction(hi) <= b


def test_reduce_batches_rejects_gaps_and_disorder():
    good = [{"n0": 1, "num": 2, "S": "[1 +/- 0.1]", "absS": "[0 +/- 1]", "g_first": "[1 +/- 0]", "g_last": "[2 +/- 0]"},
            {"n0": 3, "num": 2, "S": "[2 +/- 0.1]", "absS": "[0 +/- 1]", "g_first": "[3 +/- 0]", "g_last": "[4 +/- 0]"}]
    main, tail, ab = certify.reduce_batches(good, 4, 2)
    assert main[0] <= 1 <= main[1] and tail[0] <= 2 <= tail[1]
    with pytest.raises(certify.CertificationError):
        certify.reduce_batches(good[:1], 4, 2)                        # does not cover 1..N
    bad = [dict(good[0]), dict(good[1], g_first="[1.5 +/- 0]")]        # not ordered by height
    with pytest.raises(certify.CertificationError):
        certify.reduce_batches(bad, 4, 2)


# ------------------------------------------------------------------ GPU: certificates

@pytest.mark.gpu
def test_certificate_contains_oracle(gpu, oracle):
    data = synth.make_table(6000, seed=9)
    T0 = str(float(data.gamma[5000]) - 1e-7)
    cert = certify.certify(data, k_str="3e-9", T0_str=T0, n_hi=3000)
    N = cert["N_T0"]
    assert N == 5000 and cert["delta_lower"] is not None
    c = synth.peak2_candidate()
    vi, vf, _ = certify.v_point(synth.PEAK2_STR)
    hi, lo = oracle.k2(c, data, 3e-9, N)
    a, b = certify.ball_bounds(cert["K2"])
    x = Fraction(hi[0, 0]) + Fraction(lo[0, 0])
    assert a <= x <= b and float(b - a) < 1e-10
    main = certify.ball_bounds(cert["K2_main_(n<=3000)"])
    hm, lm = oracle.k2(c, data, 3e-9, 3000)
    assert main[0] <= Fraction(hm[0, 0]) + Fraction(lm[0, 0]) <= main[1]


@pytest.mark.gpu
def test_batched_certificate_and_cache(gpu, tmp_path):
    data = synth.make_table(3000, seed=10)
    T0 = str(float(data.gamma[2000]) - 1e-7)
    one = certify.certify(data, k_str="3e-9", T0_str=T0, n_hi=1000)
    bat = certify.certify(data, k_str="3e-9", T0_str=T0, n_hi=1000, batch=250, outdir=str(tmp_path))
    a1, b1 = certify.ball_bounds(one["K2"])
    a2, b2 = certify.ball_bounds(bat["K2"])
    assert max(a1, a2) <= min(b1, b2)                                  # the enclosures overlap
    assert len(os.listdir(tmp_path)) == 8
    # a cached payload whose key does not match is rejected (certification/test_certio.py:43-47)
    path = os.path.join(tmp_path, "00000001_250_45.json")
    d = json.load(open(path))
    d["tag"] = "other"
    json.dump(d, open(path, "w"))
    with pytest.raises(certify.CertificationError):
        certify.certify(data, k_str="3e-9", T0_str=T0, n_hi=1000, batch=250, outdir=str(tmp_path))


@pytest.mark.gpu
def test_cli_exit_codes(gpu, tmp_path):
    out = str(tmp_path / "c.json")
    assert certify.main(["--T0", "2000", "--k", "3e-9", "--out", out]) == 0
    assert json.load(open(out))["N_T0"] > 0
    assert certify.main(["--T0", "10", "--out", out]) == 1             # no zeros below T0


def test_cli_cache_only_refused():
    """certify_K2.py's zero-generation mode is outside the evaluator: a clear refusal, exit 2."""
    assert certify.main(["24", "--cache-only"]) == 2


@pytest.mark.gpu
def test_cli_reads_cache_dir(gpu, tmp_path):
    """certify_K2.py's command line ([workers] --v --k --out) over a zero_cache/ directory."""
    from mertens_bound_b200 import formats, synth
    data = synth.make_table_below(1500.0, seed=3)
    half = data.n // 2
    d = tmp_path / "zero_cache"
    d.mkdir()
    formats.write_zero_cache(str(d / f"{1:08d}_{half}_45.txt"), data.truncate(half))
    rest = synth.ZeroTableData(data.G3[half:].copy(), data.gamma[half:].copy(), data.c_re[half:].copy(),
                               data.c_im[half:].copy(), data.seed)
    formats.write_zero_cache(str(d / f"{half + 1:08d}_{data.n - half}_45.txt"), rest)
    out = str(tmp_path / "c.json")
    assert certify.main(["24", "--k", "3e-9", "--T0", "1000", "--cache-dir", str(d), "--out", out]) == 0
    cert = json.load(open(out))
    assert cert["N_T0"] == data.count_below(1000.0)
