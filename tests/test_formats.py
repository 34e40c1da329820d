"""Reference table formats: exact round trips, corruption detection, agreement with the
oracle's independent adapter."""
import os
import struct

import numpy as np
import pytest

from mertens_bound_b200 import formats, synth
from oracle.oracle import reference_format


@pytest.fixture(scope="module")
def tab():
    return synth.make_table(3000, seed=3)


def test_ghi_glo_round_trip_exact(tab):
    f = formats.ghi_glo_from_G3(tab.G3)
    G3 = formats.G3_from_ghi_glo(*f)
    assert np.array_equal(G3, tab.G3)


def test_fields_agree_with_oracle_adapter(tab):
    mine = formats.reference_fields(tab.truncate(200), exact_psi=True)
    theirs = reference_format(tab, 200, exact_psi=True)
    for k in ("ghi_lo", "ghi_hi", "glo_lo", "glo_hi", "psi_lo", "psi_hi"):
        assert np.array_equal(mine[k], theirs[k]), k


def test_glo_round_half_even_edge():
    # G with low 30 bits exactly one half: rounding to even, and back exactly
    G3 = np.array([[5, 1 << 40, (1 << 29)], [5, 1 << 40, (1 << 29) | (1 << 30)]], dtype=np.uint64)
    f = formats.ghi_glo_from_G3(G3)
    assert int(f[2][0]) & 1 == 0 and int(f[2][1]) & 1 == 0
    assert np.array_equal(formats.G3_from_ghi_glo(*f), G3)


def test_zeros_600k_round_trip(tab, tmp_path):
    p = str(tmp_path / "zeros_600k.bin")
    f = formats.reference_fields(tab, exact_psi=False)
    formats.write_zeros_600k(p, f)
    g = formats.read_zeros_600k(p)
    t2 = formats.table_from_fields(g)
    assert np.array_equal(t2.G3, tab.G3) and np.array_equal(t2.gamma, tab.gamma)
    c = tab.c_re + 1j * tab.c_im
    c2 = t2.c_re + 1j * t2.c_im
    assert np.max(np.abs(c2 - c) / np.abs(c)) < 1e-14


def test_zeros_bin_round_trip(tab, tmp_path):
    p = str(tmp_path / "zeros.bin")
    f = formats.reference_fields(tab.truncate(500), exact_psi=False)
    formats.write_zeros_bin(p, f)
    g = formats.read_zeros_bin(p)
    assert g["n"] == 500
    assert np.array_equal(formats.G3_from_ghi_glo(g["ghi_lo"], g["ghi_hi"], g["glo_lo"], g["glo_hi"]), tab.G3[:500])
    assert np.max(np.abs(g["alpha"] / f["alpha"] - 1)) < 1e-13


def test_truncated_and_inconsistent_files_rejected(tab, tmp_path):
    p = str(tmp_path / "z.bin")
    formats.write_zeros_600k(p, formats.reference_fields(tab.truncate(50), exact_psi=False))
    data = open(p, "rb").read()
    open(p, "wb").write(data[:-8])
    with pytest.raises(formats.FormatError):
        formats.read_zeros_600k(p)
    f = formats.reference_fields(tab.truncate(50), exact_psi=False)
    f["glo_lo"] = f["glo_lo"] ^ np.uint64(1 << 10)          # glo bits that ghi also carries
    with pytest.raises(formats.FormatError):
        formats.table_from_fields(f)
    q = str(tmp_path / "zb.bin")
    open(q, "wb").write(struct.pack("<i", -3))
    with pytest.raises(formats.FormatError):
        formats.read_zeros_bin(q)


def test_zero_cache_round_trip(tab, tmp_path):
    p = str(tmp_path / "00000001_100_45.txt")
    t = tab.truncate(100)
    formats.write_zero_cache(p, t)
    t2, rad = formats.read_zero_cache(p)
    d = (t2.G3[:, 2].astype(object) - t.G3[:, 2].astype(object))
    assert np.array_equal(t2.G3[:, :2], t.G3[:, :2]) and all(abs(int(x)) <= 1 for x in d)
    assert np.array_equal(t2.c_re, t.c_re) and np.array_equal(t2.c_im, t.c_im)
    # gamma radius: decimal rounding (~1e-50) plus flooring G to 2^-128 (2pi 2^-128 = 1.85e-38)
    assert np.all(rad.gamma >= 2 * np.pi * 2.0 ** -128) and np.all(rad.gamma < 1e-37)
    # c midpoints are decimal strings; storing them as FP64 adds up to half an ulp (~1e-18)
    r = formats.term_radius(rad, t2, 3.5e18)
    assert np.all(r >= 0) and np.all(r < 1e-17)


def test_parse_ball():
    assert formats.parse_ball("[14.1347 +/- 2.1e-48]") == ("14.1347", 2.1e-48)
    assert formats.parse_ball("0.5") == ("0.5", 0.0)
    with pytest.raises(ValueError):
        formats.parse_ball("[nonsense]")
