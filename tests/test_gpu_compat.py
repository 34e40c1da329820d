"""The reference-compatible entry points against the reference's own compiled evaluator
(oracle/_ref/libpath1_eval.so, built from search/path1_eval_fast.cpp) on the same inputs."""
import numpy as np
import pytest

from mertens_bound_b200 import compat, synth
from oracle.oracle import RefLib, reference_candidates, reference_format

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not RefLib.available(), reason="reference evaluator not built")]


@pytest.fixture(scope="module")
def ref_inputs(gpu, small_table):
    t = small_table.truncate(6000)
    cd = synth.make_candidates(24, seed=61)
    cd.delta[:] = np.linspace(-2e-5, 2e-5, cd.n)
    return t, cd, reference_candidates(cd), reference_format(t)


def test_compute_peak_AB_matches_reference(ref_inputs):
    t, cd, refc, reft = ref_inputs
    R = RefLib()
    A0, B0 = R.peak_AB(refc, reft)
    keys = ("alpha", "gamma", "ghi_lo", "ghi_hi", "glo_lo", "glo_hi", "psi_lo", "psi_hi")
    A, B = compat.compute_peak_AB(*refc, *(reft[k] for k in keys))
    scale = 2 * reft["alpha"][None, :]
    # same th up to an FMA contraction; cos/sin implementations differ by a few ulp
    assert np.max(np.abs(A - A0) / scale) < 1e-13
    assert np.max(np.abs(B - B0) / scale) < 1e-13


@pytest.mark.parametrize("steps", [0, 40])
def test_polish_matches_reference(ref_inputs, steps):
    t, cd, refc, reft = ref_inputs
    R = RefLib()
    A, B = R.peak_AB(refc, reft)
    w = np.exp(-3e-9 * t.gamma ** 2)
    hu0, hp0, dp0 = R.polish(A, B, t.gamma, w, 2.5e-4, steps)
    hu, hp, dp = compat.polish_peaks_with_weights(A, B, t.gamma, w, 2.5e-4, steps)
    assert np.max(np.abs(hu - hu0)) < 1e-13
    assert np.max(np.abs(hp - hp0)) < 1e-12
    assert np.max(np.abs(dp - dp0)) < 1e-9


def test_compat_void_form_reports_failure(k2lib, capfd):
    # null arrays: the void form cannot return a status; it reports on stderr and writes NaN
    out = np.zeros(4)
    k2lib.polish_peaks_with_weights(4, 10, None, None, None, None, 1e-4, 0, out.ctypes.data,
                                    out.ctypes.data, out.ctypes.data)
    assert np.all(np.isnan(out))
    assert "polish_peaks_with_weights failed" in capfd.readouterr().err
