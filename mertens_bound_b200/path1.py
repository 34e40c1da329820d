"""The per-peak polish interface of search/path1_kernel_opt.py on the GPU.

Matrix forms (same arguments and results as the reference functions):

    A, B = compute_exact_AB(table, cands)                       # compute_exact_mpfr_AB, :71-91
    h0, h, ddy = polish_single_peak(A[i], B[i], gamma, w)       # :94-147 (also 2-D: every row)
    h_unpol, h_pol, ddy_pol = fast_polish_batch(A, B, gamma, w) # fast_polish_batch_blas, :150-221

Fused forms, which compute (A_j, B_j) on the fly from the exact phase of each peak's v (+ delta)
and never form the P x N matrices:

    slot = table.add_weights(w)
    h0, h, ddy = polish_single_exact(table, cands, slot, n_zeros)
    h_unpol, h_pol, ddy_pol = fast_polish_exact(table, cands, slot, n_zeros)
    h_unpol, h_pol, ddy_pol = polish_peaks_exact(table, cands, slot, n_zeros)   # path1_eval_fast.cpp:58

Errors raise K2Error.  A peak is y = v + delta, v in 64.64 fixed point
(mertens_bound_b200.synth.Candidates).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from ._lib import check, ptr


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _cands(cands):
    vi = np.ascontiguousarray(cands.v_int, dtype=np.uint64)
    vf = np.ascontiguousarray(cands.v_frac, dtype=np.uint64)
    d = getattr(cands, "delta", None)
    d = None if d is None else _f64(d)
    if vf.shape != vi.shape or (d is not None and d.shape != vi.shape):
        raise ValueError("candidate arrays must have equal shapes")
    return vi, vf, d


def default_grid():
    """The reference's default Taylor-polish grid: 121 points on [-3e-5, 3e-5]."""
    return np.linspace(-3.0e-5, 3.0e-5, 121)


def compute_exact_AB(table, cands, n_zeros: int | None = None):
    """A, B of shape (P, n_zeros): 2 Re / 2 Im of c_j e^{i gamma_j y} from the exact phase."""
    vi, vf, d = _cands(cands)
    n = table.n if n_zeros is None else int(n_zeros)
    A = np.empty((vi.shape[0], n))
    B = np.empty((vi.shape[0], n))
    check(_lib.lib().mb_exact_AB(table.handle, vi.shape[0], ptr(vi), ptr(vf), ptr(d), n, ptr(A), ptr(B)))
    return A, B


def polish_single_peak(A, B, gamma, w, n_zeros=None, grid_hw: float = 4e-5, grid_steps: int = 40):
    """(h_unpol, h_pol, ddy_pol); floats for 1-D A/B (one peak), arrays for 2-D (one per row)."""
    A, B = _f64(A), _f64(B)
    one = A.ndim == 1
    if one:
        A, B = A[None, :], B[None, :]
    if A.shape != B.shape or A.ndim != 2:
        raise ValueError("A and B must have equal 1-D or 2-D shapes")
    P, ld = A.shape
    n = min(ld, len(gamma)) if n_zeros is None else int(n_zeros)
    if n > ld:
        raise ValueError("n_zeros exceeds the row length")
    g, ww = _f64(gamma)[:n].copy(), _f64(w)[:n].copy()
    if g.shape != (n,) or ww.shape != (n,):
        raise ValueError("gamma and w must hold n_zeros values")
    hu, hp, dp = np.empty(P), np.empty(P), np.empty(P)
    check(_lib.lib().mb_polish_single_peak(P, n, ld, ptr(A), ptr(B), ptr(g), ptr(ww), float(grid_hw),
                                           int(grid_steps), ptr(hu), ptr(hp), ptr(dp)))
    if one:
        return float(hu[0]), float(hp[0]), float(dp[0])
    return hu, hp, dp


def fast_polish_batch(A_mat, B_mat, gamma_vec, w_vec, ddy_grid=None, top: int = 25):
    """(h_unpol, h_pol, ddy_pol) for every row of A_mat/B_mat."""
    A, B = _f64(A_mat), _f64(B_mat)
    if A.shape != B.shape or A.ndim != 2:
        raise ValueError("A_mat and B_mat must be equal 2-D arrays")
    P, N = A.shape
    g, ww = _f64(gamma_vec), _f64(w_vec)
    if g.shape != (N,) or ww.shape != (N,):
        raise ValueError("gamma_vec and w_vec must have one value per column")
    grid = _f64(default_grid() if ddy_grid is None else ddy_grid)
    hu, hp, dp = np.empty(P), np.empty(P), np.empty(P)
    check(_lib.lib().mb_fast_polish_batch(P, N, ptr(A), ptr(B), ptr(g), ptr(ww), ptr(grid), grid.shape[0],
                                          int(top), ptr(hu), ptr(hp), ptr(dp)))
    return hu, hp, dp


def polish_single_exact(table, cands, weight_slot: int, n_zeros: int | None = None, grid_hw: float = 4e-5,
                        grid_steps: int = 40):
    """polish_single_peak for every candidate, (A, B) computed on the fly."""
    vi, vf, d = _cands(cands)
    P = vi.shape[0]
    n = table.n if n_zeros is None else int(n_zeros)
    hu, hp, dp = np.empty(P), np.empty(P), np.empty(P)
    check(_lib.lib().mb_polish_single_exact(table.handle, P, ptr(vi), ptr(vf), ptr(d), n, int(weight_slot),
                                            float(grid_hw), int(grid_steps), ptr(hu), ptr(hp), ptr(dp)))
    return hu, hp, dp


def fast_polish_exact(table, cands, weight_slot: int, n_zeros: int | None = None, ddy_grid=None, top: int = 25):
    """fast_polish_batch for every candidate, (A, B) computed on the fly."""
    vi, vf, d = _cands(cands)
    P = vi.shape[0]
    n = table.n if n_zeros is None else int(n_zeros)
    grid = _f64(default_grid() if ddy_grid is None else ddy_grid)
    hu, hp, dp = np.empty(P), np.empty(P), np.empty(P)
    check(_lib.lib().mb_fast_polish_exact(table.handle, P, ptr(vi), ptr(vf), ptr(d), n, int(weight_slot),
                                          ptr(grid), grid.shape[0], int(top), ptr(hu), ptr(hp), ptr(dp)))
    return hu, hp, dp


def polish_peaks_exact(table, cands, weight_slot: int, n_zeros: int | None = None,
                       grid_half_width: float = 2.5e-4, grid_steps: int = 40):
    """polish_peaks_with_weights (search/path1_eval_fast.cpp:58-143) for every candidate, (A, B)
    computed on the fly; the defaults are the search drivers' settings (eval_tech1_600k.py:262)."""
    vi, vf, d = _cands(cands)
    P = vi.shape[0]
    n = table.n if n_zeros is None else int(n_zeros)
    hu, hp, dp = np.empty(P), np.empty(P), np.empty(P)
    check(_lib.lib().mb_polish_peaks_exact(table.handle, P, ptr(vi), ptr(vf), ptr(d), n, int(weight_slot),
                                           float(grid_half_width), int(grid_steps), ptr(hu), ptr(hp), ptr(dp)))
    return hu, hp, dp


def polish_peaks_weights(table, cands, weight_slots, n_zeros: int | None = None,
                         grid_half_width: float = 2.5e-4, grid_steps: int = 40):
    """polish_peaks_exact under several registered weight vectors at once: (h_unpol, h_pol,
    ddy_pol), each of shape (len(weight_slots), P).  The exact (A, B) is built once in device
    memory and read by every weight's polish (search/eval_tech1_600k.py:216-273)."""
    vi, vf, d = _cands(cands)
    P = vi.shape[0]
    n = table.n if n_zeros is None else int(n_zeros)
    slots = np.ascontiguousarray(weight_slots, dtype=np.int32)
    W = slots.shape[0]
    hu, hp, dp = np.empty((W, P)), np.empty((W, P)), np.empty((W, P))
    check(_lib.lib().mb_polish_peaks_weights(table.handle, P, ptr(vi), ptr(vf), ptr(d), n, W, ptr(slots),
                                             float(grid_half_width), int(grid_steps), ptr(hu), ptr(hp), ptr(dp)))
    return hu, hp, dp
