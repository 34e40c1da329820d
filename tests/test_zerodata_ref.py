"""The enumerators' leaf screen and hit polish pinned to the reference itself: the committed
fixture tests/golden/zerodata_ref.json holds the decisions and values of the reference's own
ZeroData (search/fast_mertens_enum.cpp:27-277, compiled from its source into
oracle/_ref/libzerodata_ref.so by oracle/Makefile through oracle/zerodata_ref.cpp).  Here (CPU):
the fixture is what that library gives, and the oracle's two restatements reproduce it --
Oracle.fast_screen (the C restatement of ZeroData::fast_screen, :108-142) and
oracle.zerodata_polish (the numpy restatement of ZeroData::polish, :145-276)."""
import hashlib
import json
import os

import numpy as np
import pytest

from mertens_bound_b200 import formats, synth

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = json.load(open(os.path.join(HERE, "golden", "zerodata_ref.json")))
MASK64 = (1 << 64) - 1
ENUM_THRESHOLDS = (0.895, 0.915, 0.945)      # fast_mertens_enum.cpp:177,203,236


def table():
    t = synth.enumerator_table(FIX["table"]["n"], FIX["table"]["seed"], FIX["table"]["c_scale"])
    h = hashlib.sha256()
    for a in (t.G3, t.gamma, t.c_re, t.c_im):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest() == FIX["table"]["sha256"], "the synthetic generator changed"
    return t


def leaves():
    x = synth.leaves_x(FIX["leaves"]["count"], FIX["leaves"]["seed"])
    xs = np.array([[v & MASK64, v >> 64] for v in x], np.uint64)
    assert hashlib.sha256(xs.tobytes()).hexdigest() == FIX["leaves"]["sha256"]
    return x, np.ascontiguousarray(xs[:, 0]), np.ascontiguousarray(xs[:, 1])


def fixture_pass():
    n = FIX["leaves"]["count"]
    return np.unpackbits(np.frombuffer(bytes.fromhex(FIX["screen_pass_packbits_hex"]), np.uint8))[:n]


@pytest.fixture(scope="module")
def reft():
    from oracle.oracle import reference_format
    t = table()
    f = reference_format(t, exact_psi=True)
    f["two_astar"] = 2.0 * f["alpha"] * np.exp(-formats.ZEROS_BIN_K * f["gamma"] ** 2)
    return t, f


def test_fixture_is_the_reference(tmp_path, reft, oracle):
    """The reference's ZeroData, run here, gives the committed decisions and polish values."""
    from oracle.oracle import ZeroDataRef
    if not ZeroDataRef.available():
        pytest.skip("oracle/_ref/libzerodata_ref.so not built (reference source absent)")
    t, f = reft
    path = str(tmp_path / "zeros.bin")
    formats.write_zeros_bin(path, f)
    Z = ZeroDataRef(path)
    x, x_lo, x_hi = leaves()
    assert np.array_equal(Z.fast_screen(x_lo, x_hi), fixture_pass())
    sel = np.array([p["leaf"] for p in FIX["polish"]])
    h, dy = Z.polish(x_lo[sel], x_hi[sel])
    assert np.array_equal(h, [p["h"] for p in FIX["polish"]])
    assert np.array_equal(dy, [p["dy"] for p in FIX["polish"]])
    Z.close()


def test_fixture_exercises_both_sides():
    p = fixture_pass()
    assert 200 < p.sum() < len(p) - 200
    h = np.abs([q["h"] for q in FIX["polish"]])
    assert np.sum(h >= ENUM_THRESHOLDS[2]) >= 30 and np.sum(h < ENUM_THRESHOLDS[0]) >= 3


def test_oracle_fast_screen_matches_reference(reft, oracle):
    t, f = reft
    x, x_lo, x_hi = leaves()
    got = oracle.fast_screen(x_lo, x_hi, f, f["two_astar"])
    assert np.array_equal(got, fixture_pass())


def test_zerodata_polish_restatement_matches_reference(reft, oracle):
    from oracle.oracle import zerodata_polish
    t, f = reft
    x, x_lo, x_hi = leaves()
    sel = np.array([p["leaf"] for p in FIX["polish"]])
    refc = (x_lo[sel], x_hi[sel], np.zeros(len(sel)))
    _, _, top = oracle.ref_peak_AB(refc, f, want_top=True)
    for i, p in enumerate(FIX["polish"]):
        h, dy = zerodata_polish(top[i].view(np.int64), f["two_astar"], f["gamma"], thresholds=ENUM_THRESHOLDS)
        assert dy == pytest.approx(p["dy"], abs=1e-15), (i, dy, p["dy"])
        assert h == pytest.approx(p["h"], rel=1e-12, abs=1e-13), (i, h, p["h"])
