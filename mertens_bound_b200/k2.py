"""Python host API of the B200 K2 evaluator.

    table = ZeroTable(G3, c_re, c_im, gamma)          # upload + validate once
    val, dd, dk = k2_plain(table, cands, k=3e-9, T=3e5)

K2(v,T,k) = 2 sum_{gamma<T} exp(-k gamma^2) Re(c e^{i gamma v}); dd = dK2/ddelta, dk = dK2/dk.
Candidates are 64.64 fixed point (v_int, v_frac) plus an FP64 offset delta
(mertens_bound_b200.synth.Candidates).
"""
from __future__ import annotations

import ctypes as C
import hashlib
import math
import weakref

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

    def add_weights(self, w) -> int:
        """Register a per-zero weight vector (length n) with the table; returns its slot.

        A plan group that names the slot sums 2 w_j Re(c_j e^{i gamma_j v}) instead of the
        Gaussian exp(-k gamma_j^2) weight.
        """
        w = _f64(w)
        if w.shape != (self.n,):
            raise ValueError(f"weights must have shape ({self.n},)")
        key = hashlib.sha1(w.tobytes()).hexdigest()      # a vector registered before keeps its slot
        cache = self.__dict__.setdefault("_weight_slots", {})
        if key in cache:
            return cache[key]
        slot = C.c_int()
        check(_lib.lib().mb_table_add_weights(self.handle, ptr(w), self.n, C.byref(slot)))
        cache[key] = slot.value
        return slot.value

    def count_below(self, T: float) -> int:
        out = C.c_int64()
        check(_lib.lib().mb_table_count_below(self.handle, float(T), C.byref(out)))
        return out.value

    def close(self):
        """Free the device table, closing first any plan made on it that is still open (the
        library refuses to free a table under live plans)."""
        if getattr(self, "_h", None) is not None:
            for plan in list(self.__dict__.get("_plans", ())):
                plan.close()
            check(_lib.lib().mb_table_destroy(self._h))
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


class Plan:
    """A batched evaluation plan: groups of candidates, each at its own (k, T).

    counts[g] consecutive candidates form group g.  tol is the a-priori bound on |K2 error|
    per candidate that fixes each group's heavy/light tier boundary.  weights[g], if given, is a
    slot from ZeroTable.add_weights (or -1 for the Gaussian exp(-k_g gamma^2)).
    """

    def __init__(self, table: ZeroTable, counts, ks, Ts, tol: float = 1e-10, weights=None):
        counts = np.ascontiguousarray(counts, dtype=np.int64)
        ks = np.ascontiguousarray(ks, dtype=np.float64)
        Ts = np.ascontiguousarray(Ts, dtype=np.float64)
        if not (counts.shape == ks.shape == Ts.shape) or counts.ndim != 1:
            raise ValueError("counts, ks, Ts must be 1-D of equal length")
        h = C.c_void_p()
        if weights is None:
            check(_lib.lib().mb_plan_create(table.handle, counts.shape[0], ptr(counts), ptr(ks), ptr(Ts),
                                            float(tol), C.byref(h)))
        else:
            weights = np.ascontiguousarray(weights, dtype=np.int32)
            if weights.shape != counts.shape:
                raise ValueError("weights must name one slot per group")
            check(_lib.lib().mb_plan_create_weighted(table.handle, counts.shape[0], ptr(counts), ptr(ks),
                                                     ptr(Ts), ptr(weights), float(tol), C.byref(h)))
        self._h = h
        self.table = table
        table.__dict__.setdefault("_plans", weakref.WeakSet()).add(self)
        self.counts, self.ks, self.Ts, self.tol = counts, ks, Ts, tol
        self.P = int(counts.sum())

    @property
    def handle(self):
        if self._h is None:
            raise ValueError("plan is closed")
        return self._h

    def set_shape(self, g: int, cpt: int, nzw: int, heavy_chunk: int = 0, light_chunk: int = 0):
        check(_lib.lib().mb_plan_set_shape(self.handle, g, cpt, nzw, heavy_chunk, light_chunk))

    def set_skip(self, skip_frac: float):
        """Skip each group's negligible tail of zeros, giving it skip_frac (<= 0.25) of tol."""
        check(_lib.lib().mb_plan_set_skip(self.handle, float(skip_frac)))

    def configure(self, light_cpt: int, nzw_shift: int, chunk_scale: float):
        check(_lib.lib().mb_plan_configure(self.handle, int(light_cpt), int(nzw_shift), float(chunk_scale)))
        self.config = (int(light_cpt), int(nzw_shift), float(chunk_scale))

    def set_schedule(self, schedule: int):
        """0: the two tier kernels run concurrently (heavy persistent kernel on a side stream);
        1: one persistent kernel runs both tiers' items, heavy first; 2: the same kernel with all
        items ordered by estimated cost, largest first; 3: the same kernel with one queue per
        tier, the first CTA on each SM pulling heavy items and the second light items."""
        check(_lib.lib().mb_plan_set_schedule(self.handle, int(schedule)))

    def schedule(self) -> int:
        s = C.c_int()
        check(_lib.lib().mb_plan_schedule(self.handle, C.byref(s)))
        return s.value

    def time(self, reps: int = 3) -> float:
        """Median device milliseconds of one run (synthetic candidates)."""
        ms = C.c_double()
        check(_lib.lib().mb_plan_time(self.handle, int(reps), C.byref(ms)))
        return ms.value

    def tier_terms(self):
        h, l = C.c_double(), C.c_double()
        check(_lib.lib().mb_plan_tier_terms(self.handle, C.byref(h), C.byref(l)))
        return h.value, l.value

    def info(self):
        """P, zero_terms, n_items and light_form: "fused" (the light tier's one-FMA fraction product,
        every zero of the table below gamma = 3.29e6) or "split"."""
        P, zt, ni, fu = C.c_int64(), C.c_double(), C.c_int(), C.c_int()
        check(_lib.lib().mb_plan_info(self.handle, C.byref(P), C.byref(zt), C.byref(ni)))
        check(_lib.lib().mb_plan_light_form(self.handle, C.byref(fu)))
        return {"P": P.value, "zero_terms": zt.value, "n_items": ni.value,
                "light_form": "fused" if fu.value else "split"}

    def group_info(self, g: int):
        nT, nh, eb, sa = C.c_int64(), C.c_int64(), C.c_double(), C.c_double()
        ne, bd, bk = C.c_int64(), C.c_double(), C.c_double()
        check(_lib.lib().mb_plan_group_info(self.handle, g, C.byref(nT), C.byref(nh), C.byref(eb), C.byref(sa)))
        check(_lib.lib().mb_plan_group_zeros(self.handle, g, C.byref(ne)))
        check(_lib.lib().mb_plan_group_bounds(self.handle, g, None, C.byref(bd), C.byref(bk)))
        return {"n_T": nT.value, "n_eval": ne.value, "n_heavy": nh.value, "err_bound": eb.value,
                "err_bound_dd": bd.value, "err_bound_dk": bk.value, "sum_abs": sa.value}

    def run(self, cands):
        """Host arrays in, host arrays out (graph replay through pinned staging)."""
        vi, vf, d = _cand_arrays(cands)
        if vi.shape[0] != self.P:
            raise ValueError(f"plan expects {self.P} candidates, got {vi.shape[0]}")
        val, dd, dk = np.empty(self.P), np.empty(self.P), np.empty(self.P)
        check(_lib.lib().mb_plan_run(self.handle, ptr(vi), ptr(vf), ptr(d), ptr(val), ptr(dd), ptr(dk)))
        return val, dd, dk

    def run_dev(self, d_vi: int, d_vf: int, d_delta, d_val: int, d_dd: int, d_dk: int, stream: int = 0):
        """Device pointers (ints), asynchronous on `stream`."""
        check(_lib.lib().mb_plan_run_dev(self.handle, d_vi, d_vf, d_delta, d_val, d_dd, d_dk, stream))

    def close(self):
        if getattr(self, "_h", None) is not None:
            _lib.lib().mb_plan_destroy(self._h)
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


def k2_certified(table: ZeroTable, cands, k: float, T: float = math.inf, v_rad=None, term_rad=None):
    """Rigorous enclosure [lo, hi] of K2 at v = v_int + v_frac 2^-64 (delta must be zero or
    absent; widen with v_rad instead), plus an upper bound of sum 2 w |c|."""
    vi, vf, d = _cand_arrays(cands)
    if d is not None and np.any(d != 0):
        raise ValueError("the certified evaluation takes exact 64.64 points; pass offsets as v_rad")
    P = vi.shape[0]
    vr = None if v_rad is None else _f64(np.broadcast_to(v_rad, (P,)))
    n_use = table.count_below(T)
    tr = None if term_rad is None else _f64(term_rad)
    if tr is not None and tr.shape != (n_use,):
        raise ValueError(f"term_rad must have count_below(T) = {n_use} entries")
    lo, hi, ab = np.empty(P), np.empty(P), np.empty(P)
    check(_lib.lib().mb_k2_certified(table.handle, P, ptr(vi), ptr(vf), ptr(vr), float(k), float(T), ptr(tr),
                                     ptr(lo), ptr(hi), ptr(ab)))
    return lo, hi, ab


def k2_certified_grad(table: ZeroTable, cands, k: float, T: float = math.inf, v_rad=None, term_rad=None,
                      k_hi: float | None = None):
    """Rigorous enclosures of K2, dK2/ddelta and dK2/dk at v = v_int + v_frac 2^-64 (widened by
    v_rad), for k in [k, k_hi] (k_hi defaults to k): returns lo, hi of shape (3, P), rows
    (K2, dK2/ddelta, dK2/dk)."""
    vi, vf, d = _cand_arrays(cands)
    if d is not None and np.any(d != 0):
        raise ValueError("the certified evaluation takes exact 64.64 points; pass offsets as v_rad")
    P = vi.shape[0]
    vr = None if v_rad is None else _f64(np.broadcast_to(v_rad, (P,)))
    n_use = table.count_below(T)
    tr = None if term_rad is None else _f64(term_rad)
    if tr is not None and tr.shape != (n_use,):
        raise ValueError(f"term_rad must have count_below(T) = {n_use} entries")
    lo, hi = np.empty((3, P)), np.empty((3, P))
    check(_lib.lib().mb_k2_certified_grad_range(table.handle, P, ptr(vi), ptr(vf), ptr(vr), float(k),
                                                float(k if k_hi is None else k_hi), 0, n_use, ptr(tr), ptr(lo),
                                                ptr(hi)))
    return lo, hi


def k2_fast(table: ZeroTable, cands, k: float, T: float = math.inf, tol: float = 1e-10):
    """Chosen-form K2, dK2/ddelta, dK2/dk and the a-priori error bound (one group)."""
    vi, vf, d = _cand_arrays(cands)
    P = vi.shape[0]
    val, dd, dk = np.empty(P), np.empty(P), np.empty(P)
    eb = C.c_double()
    check(_lib.lib().mb_k2_fast(table.handle, P, ptr(vi), ptr(vf), ptr(d), float(k), float(T), float(tol),
                                ptr(val), ptr(dd), ptr(dk), C.byref(eb)))
    return val, dd, dk, eb.value
