"""The reference's evaluator interface (search/path1_eval_fast.cpp) on the GPU.

    A, B = compute_peak_AB(x_lo, x_hi, dy0, alpha, gamma, ghi_lo, ghi_hi, glo_lo, glo_hi,
                           psi_lo, psi_hi)
    h_unpol, h_pol, ddy_pol = polish_peaks_with_weights(A, B, gamma, w, grid_half_width, grid_steps)

Argument meaning follows the reference exactly (see its callers,
search/eval_tech1_600k.py:201-273): x = floor(y 2^30) as a u128 split into (x_lo, x_hi),
dy0 the FP64 remainder, and the zero table in the zeros_600k.bin field set
(mertens_bound_b200.formats reads and writes it).  Errors raise K2Error (the reference has no
error channel).  The library also exports the two functions under their original C names, so
the reference's own ctypes drivers can load libmertens_k2.so unchanged.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from ._lib import check, ptr


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def compute_peak_AB(x_lo, x_hi, dy0, alpha, gamma, ghi_lo, ghi_hi, glo_lo, glo_hi, psi_lo, psi_hi):
    x_lo, x_hi, dy0 = _u64(x_lo), _u64(x_hi), _f64(dy0)
    zs = [_f64(alpha), _f64(gamma)] + [_u64(a) for a in (ghi_lo, ghi_hi, glo_lo, glo_hi, psi_lo, psi_hi)]
    P, N = x_lo.shape[0], zs[0].shape[0]
    if any(z.shape != (N,) for z in zs) or x_hi.shape != (P,) or dy0.shape != (P,):
        raise ValueError("array shapes do not match")
    A = np.empty((P, N))
    B = np.empty((P, N))
    check(_lib.lib().mb_compute_peak_AB(P, ptr(x_lo), ptr(x_hi), ptr(dy0), N, *[ptr(z) for z in zs],
                                        ptr(A), ptr(B)))
    return A, B


def polish_peaks_with_weights(A, B, gamma, w, grid_half_width: float, grid_steps: int):
    A, B = _f64(A), _f64(B)
    P, N = A.shape
    g = _f64(gamma)[:N].copy()
    ww = _f64(w)[:N].copy()
    if B.shape != A.shape or g.shape != (N,) or ww.shape != (N,):
        raise ValueError("array shapes do not match")
    hu, hp, dp = np.empty(P), np.empty(P), np.empty(P)
    check(_lib.lib().mb_polish_peaks_with_weights(P, N, ptr(A), ptr(B), ptr(g), ptr(ww), float(grid_half_width),
                                                  int(grid_steps), ptr(hu), ptr(hp), ptr(dp)))
    return hu, hp, dp
