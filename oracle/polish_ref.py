"""numpy restatement of the per-peak polishes of search/path1_kernel_opt.py -- TEST
INFRASTRUCTURE ONLY (the checker for mertens_bound_b200.path1; never the product path).

The reference module cannot be imported here (it imports gmpy2 and loads its shared library at
import time), so its two polish functions are restated from their published behaviour:

  polish_single_peak      search/path1_kernel_opt.py:94-147
  fast_polish_batch_blas  search/path1_kernel_opt.py:150-221

and the FP64 grid of search/polish.py's scan (:50-72; its mpfr phase reduction is the caller's):

  scan_grid

Both work on caller A/B rows; the numerics are plain FP64 numpy, as in the reference.  The
restatement differs from the reference only in the top-peak order on exact ties of |h_pol|
(index order here; numpy's default argsort leaves it unspecified).
"""
from __future__ import annotations

import math

import numpy as np


def _newton(Ap, Bp, gp, wp, ddy, iters, clamp, tol):
    for _ in range(iters):
        th = gp * ddy
        c = np.cos(th)
        s = np.sin(th)
        val = Ap * c - Bp * s
        dval = gp * (-Ap * s - Bp * c)
        ddval = -(gp * gp) * val
        fp = float(np.dot(wp, dval))
        fpp = float(np.dot(wp, ddval))
        if abs(fpp) > 1e-12:
            step = max(-clamp, min(clamp, fp / fpp))
            ddy -= step
            if abs(step) < tol:
                break
        else:
            break
    return ddy


def _h(Ap, Bp, gp, wp, ddy):
    th = gp * ddy
    return float(np.dot(wp, Ap * np.cos(th) - Bp * np.sin(th)))


def polish_single_peak(A, B, gamma, w, n_zeros=None, grid_hw=4e-5, grid_steps=40):
    """(h_unpol, h_pol, ddy_pol) of one peak (path1_kernel_opt.py:94-147)."""
    n = len(gamma) if n_zeros is None else n_zeros
    Ap, Bp, gp, wp = A[:n], B[:n], gamma[:n], w[:n]
    wA, wB = wp * Ap, wp * Bp
    h0 = float(np.sum(wA))
    starts = [0.0]
    if grid_steps > 0:
        ddys = np.linspace(-grid_hw, grid_hw, 2 * grid_steps + 1)
        th = np.outer(ddys, gp)
        vals = np.cos(th) @ wA - np.sin(th) @ wB
        starts.append(float(ddys[int(np.argmax(np.abs(vals)))]))
    best_h, best_ddy = h0, 0.0
    for d0 in starts:
        ddy = _newton(Ap, Bp, gp, wp, d0, 8, 2e-5, 1e-14)
        h = _h(Ap, Bp, gp, wp, ddy)
        if abs(h) > abs(best_h):
            best_h, best_ddy = h, ddy
    return h0, best_h, best_ddy


def fast_polish_batch(A_mat, B_mat, gamma_vec, w_vec, ddy_grid=None, top=25):
    """(h_unpol, h_pol, ddy_pol) of every peak (path1_kernel_opt.py:150-221)."""
    if ddy_grid is None:
        ddy_grid = np.linspace(-3.0e-5, 3.0e-5, 121)
    u = gamma_vec * 1.0e-4
    z = ddy_grid * 1.0e4
    U_cos = np.stack([w_vec * u ** (2 * m) * ((-1.0) ** m / math.factorial(2 * m)) for m in range(9)], axis=1)
    U_sin = np.stack([w_vec * u ** (2 * m + 1) * ((-1.0) ** m / math.factorial(2 * m + 1)) for m in range(8)],
                     axis=1)
    Z_cos = np.stack([z ** (2 * m) for m in range(9)])
    Z_sin = np.stack([z ** (2 * m + 1) for m in range(8)])
    C_mom = A_mat @ U_cos
    S_mom = B_mat @ U_sin
    vals = C_mom @ Z_cos - S_mom @ Z_sin
    h_unpol = C_mom[:, 0].copy()
    best = np.argmax(np.abs(vals), axis=1)
    rows = np.arange(A_mat.shape[0])
    h_pol = vals[rows, best]
    ddy_pol = ddy_grid[best].astype(np.float64)
    order = sorted(range(len(h_pol)), key=lambda i: (-abs(h_pol[i]), i))[:top]
    for i in order:
        ddy = _newton(A_mat[i], B_mat[i], gamma_vec, w_vec, float(ddy_pol[i]), 4, 1e-5, 1e-13)
        h = _h(A_mat[i], B_mat[i], gamma_vec, w_vec, ddy)
        if abs(h) > abs(h_unpol[i]):
            h_pol[i], ddy_pol[i] = h, ddy
        else:
            h_pol[i], ddy_pol[i] = h_unpol[i], 0.0
    return h_unpol, h_pol, ddy_pol


def scan_grid(phi, dphi, gre, gim, m0, m1, chunk=4000):
    """h(y0 + m step) for m in [m0, m1) as search/polish.py:60-66 forms it: angles
    phi + m dphi in FP64 (phi = gamma y0 mod 2pi, dphi = gamma step mod 2pi), chunks of `chunk`
    grid points, h = 2 sum(gre cos - gim sin) with (gre, gim) = e^{-k gamma^2} (Re c, Im c)."""
    out = []
    for a in range(m0, m1, chunk):
        b = min(a + chunk, m1)
        m = np.arange(a, b, dtype=np.float64)[:, None]
        ang = phi[None, :] + m * dphi[None, :]
        out.append(2.0 * np.sum(gre * np.cos(ang) - gim * np.sin(ang), axis=1))
    return np.concatenate(out) if out else np.empty(0)
