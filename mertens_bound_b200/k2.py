"""Python host API of the B200 K2 evaluator.

    table = ZeroTable(G3, c_re, c_im, gamma)          # upload + validate once
    val, dd, dk = k2_plain(table, cands, k=3e-9, T=3e5)

K2(v,T,k) = 2 sum_{gamma<T} exp(-k gamma^2) Re(c e^{i gamma v}); dd = dK2/ddelta, dk = dK2/dk.
Candidates are 64.64 fixed point (v_int, v_frac) plus an FP64 offset delta
(mertens_bound_b200.synth.Candidates).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import check, ptr


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class ZeroTable:
    """A zero table resident on one GPU (G = gamma/2pi in 64.128 fixed point, c, gamma)."""

    def __init__(self, G3, c_re, c_im, gamma, device: int = 0):
        G3 = _u64(G3)
        if G3.ndim != 2 or G3.shape[1] != 3:
            raise ValueError("G3 must have shape (n, 3)")
        c_re, c_im, gamma = _f64(c_re), _f64(c_im), _f64(gamma)
        n = G3.shape[0]
        if not (c_re.shape == c_im.shape == gamma.shape == (n,)):
            raise ValueError("c_re, c_im, gamma must have shape (n,)")
        h = C.c_void_p()
        check(_lib.lib().mb_table_create(ptr(G3), ptr(c_re), ptr(c_im), ptr(gamma), n, device, C.byref(h)))
        self._h = h
        self.n = n
        self.device = device
        self.gamma = gamma          # host copy (cutoffs, error planning)
        self.alpha = np.hypot(c_re, c_im)

    @classmethod
    def from_data(cls, data, device: int = 0) -> "ZeroTable":
        return cls(data.G3, data.c_re, data.c_im, data.gamma, device=device)

    @property
    def handle(self):
        if self._h is None:
            raise ValueError("table is closed")
        return self._h

    def count_below(self, T: float) -> int:
        out = C.c_int64()
        check(_lib.lib().mb_table_count_below(self.handle, float(T), C.byref(out)))
        return out.value

    def close(self):
        if getattr(self, "_h", None) is not None:
            _lib.lib().mb_table_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _cand_arrays(cands):
    vi, vf = _u64(cands.v_int), _u64(cands.v_frac)
    d = getattr(cands, "delta", None)
    d = None if d is None else _f64(d)
    if vi.shape != vf.shape or (d is not None and d.shape != vi.shape):
        raise ValueError("candidate arrays must have equal shapes")
    return vi, vf, d


def phase128(table: ZeroTable, cands, n_zeros: int | None = None):
    """Exact floor(frac(v G_j) 2^128) as (hi, lo) uint64 arrays of shape (P, n_zeros)."""
    vi, vf, _ = _cand_arrays(cands)
    n = table.n if n_zeros is None else int(n_zeros)
    hi = np.empty((vi.shape[0], n), dtype=np.uint64)
    lo = np.empty_like(hi)
    check(_lib.lib().mb_phase128(table.handle, vi.shape[0], ptr(vi), ptr(vf), n, ptr(hi), ptr(lo)))
    return hi, lo


def k2_plain(table: ZeroTable, cands, k: float, T: float = math.inf):
    """Plain FP64 K2, dK2/ddelta and dK2/dk for every candidate (host arrays)."""
    vi, vf, d = _cand_arrays(cands)
    P = vi.shape[0]
    val, dd, dk = np.empty(P), np.empty(P), np.empty(P)
    check(_lib.lib().mb_k2_plain(table.handle, P, ptr(vi), ptr(vf), ptr(d), float(k), float(T),
                                 ptr(val), ptr(dd), ptr(dk)))
    return val, dd, dk
