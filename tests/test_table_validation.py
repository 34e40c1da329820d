"""Corrupt or inconsistent zero tables are rejected through the C-ABI with MB_ERR_TABLE and a
message, before any device work (runs without a GPU).  The reference's loaders check nothing
(search/eval_tech1_600k.py:38-50); certify_K2.py:82-84 rejects unordered or non-finite caches."""
import numpy as np
import pytest

from mertens_bound_b200 import k2, synth
from mertens_bound_b200._lib import K2Error


@pytest.fixture
def data():
    return synth.make_table(50, seed=21)


def _create(d):
    return k2.ZeroTable(d.G3, d.c_re, d.c_im, d.gamma)


@pytest.mark.parametrize("corrupt, msg", [
    (lambda d: d.gamma.__setitem__(10, d.gamma[9]), "not strictly increasing"),
    (lambda d: d.gamma.__setitem__(5, np.nan), "not finite and positive"),
    (lambda d: d.gamma.__setitem__(0, -1.0), "not finite and positive"),
    (lambda d: d.c_re.__setitem__(7, np.inf), "non-finite c"),
    (lambda d: d.c_im.__setitem__(8, np.nan), "non-finite c"),
    (lambda d: d.G3.__setitem__((3, 0), 1 << 33), "integer part"),
    (lambda d: d.gamma.__setitem__(20, d.gamma[20] * (1 + 1e-12)), "exceeds 4 ulp"),
])
def test_corrupt_tables_rejected(k2lib, data, corrupt, msg):
    corrupt(data)
    with pytest.raises(K2Error) as e:
        _create(data)
    assert e.value.status == -2 and msg in str(e.value)


def test_shape_mismatch_rejected_on_host(data):
    with pytest.raises(ValueError):
        k2.ZeroTable(data.G3[:-1], data.c_re, data.c_im, data.gamma)


def test_bad_arguments_are_status_codes(k2lib):
    import ctypes as C
    out = C.c_void_p()
    assert k2lib.mb_table_create(None, None, None, None, 0, 0, C.byref(out)) == -1
    assert k2lib.mb_plan_create(None, 1, None, None, None, 1e-10, C.byref(out)) == -1
    assert k2lib.mb_k2_plain(None, 1, None, None, None, 3e-9, 1.0, None, None, None) == -1
    assert k2lib.mb_k2_certified(None, 1, None, None, None, 3e-9, 1.0, None, None, None, None) == -1
