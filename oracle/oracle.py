"""CPU oracle for the K2 evaluator -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference leg may
import this module.  It is the checker, never the thing measured or shipped.

Contents
  * phase128_bigint     -- exact floor(frac(v G) 2^128) with Python integers (the definition).
  * Oracle              -- binding of _build/liboracle.so (k2_oracle.c): exact phase and the
                           K2 value/gradient sums in binary128.
  * reference_format    -- the synthetic table and candidates in the reference's layout
                           (search/path1_build_zeros_100k.py:102-104: ghi = rint(G 2^146) mod 2^128,
                           glo = rint(G 2^98), psi = rint(((-arg c / 2pi) mod 1) 2^128), alpha = |c|;
                           x = floor(v 2^30) as u128 with the remaining fraction in dy0,
                           search/eval_tech1_600k.py:213-215).
  * polish_ref          -- (module oracle.polish_ref) numpy restatement of the per-peak polishes of
                           search/path1_kernel_opt.py.
  * Oracle.fast_screen  -- restated ZeroData::fast_screen (search/fast_mertens_enum.cpp:108-142).
  * RefLib              -- binding of _ref/libpath1_eval.so, the reference's own evaluator
                           compiled from search/path1_eval_fast.cpp (see Makefile).
  * ZeroDataRef         -- binding of _ref/libzerodata_ref.so, the reference enumerator's own
                           ZeroData (search/fast_mertens_enum.cpp:27-277: load, fast_screen,
                           polish) behind the harness zerodata_ref.cpp.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libpath1_eval.so")
ZD_SO = os.path.join(HERE, "_ref", "libzerodata_ref.so")
MASK64 = (1 << 64) - 1
MASK128 = (1 << 128) - 1


def build() -> None:
    """Compile the oracle (and the reference evaluator when its source is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True, capture_output=True)


# ------------------------------------------------------------------ exact phase (definition)

def phase128_bigint(vi: int, vf: int, g: tuple[int, int, int]) -> tuple[int, int]:
    """floor(frac(v G) 2^128) for v = vi + vf 2^-64, G = g0 + g1 2^-64 + g2 2^-128."""
    V = (int(vi) << 64) | int(vf)
    Gf = (int(g[0]) << 128) | (int(g[1]) << 64) | int(g[2])
    ph = ((V * Gf) >> 64) & MASK128
    return ph >> 64, ph & MASK64


# ------------------------------------------------------------------ C oracle

def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Oracle:
    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.orc_phase128.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_k2_quad.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]
        L.orc_k2_quad_w.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]
        L.orc_exact_AB.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_abs_sum.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]
        L.orc_abs_sum.restype = C.c_double
        L.orc_gamma_from_G.argtypes = [C.c_int64, C.c_void_p, C.c_void_p]
        L.orc_ref_peak_AB.argtypes = [C.c_int] + [C.c_void_p] * 3 + [C.c_int] + [C.c_void_p] * 11
        L.orc_ref_polish.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 4 + [C.c_double, C.c_int] + [C.c_void_p] * 3
        L.orc_fast_screen.argtypes = [C.c_int64] + [C.c_void_p] * 11
        L.orc_fast_screen.restype = C.c_int64
        self.L = L

    def phase128(self, cands, G3, n=None):
        vi = np.ascontiguousarray(cands.v_int, dtype=np.uint64)
        vf = np.ascontiguousarray(cands.v_frac, dtype=np.uint64)
        G3 = np.ascontiguousarray(G3 if n is None else G3[:n], dtype=np.uint64)
        P, N = vi.shape[0], G3.shape[0]
        hi = np.empty((P, N), dtype=np.uint64)
        lo = np.empty((P, N), dtype=np.uint64)
        self.L.orc_phase128(P, _p(vi), _p(vf), N, _p(G3), _p(hi), _p(lo))
        return hi, lo

    def k2(self, cands, table, k: float, n_use: int, weights=None):
        """(val, dd, dk) in binary128, returned as (P, 3) hi parts and (P, 3) lo parts.

        weights (length >= n_use) replaces exp(-k gamma^2) per zero when given."""
        vi = np.ascontiguousarray(cands.v_int, dtype=np.uint64)
        vf = np.ascontiguousarray(cands.v_frac, dtype=np.uint64)
        d = np.ascontiguousarray(cands.delta, dtype=np.float64)
        P = vi.shape[0]
        out = np.empty((P, 6), dtype=np.float64)
        G3 = np.ascontiguousarray(table.G3, dtype=np.uint64)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        if w is not None and w.shape[0] < n_use:
            raise ValueError("weights shorter than n_use")
        self.L.orc_k2_quad_w(P, _p(vi), _p(vf), _p(d), int(n_use), _p(G3), _p(np.ascontiguousarray(table.c_re)),
                             _p(np.ascontiguousarray(table.c_im)), float(k), None if w is None else _p(w), _p(out))
        return out[:, 0::2].copy(), out[:, 1::2].copy()

    def exact_AB(self, cands, table, n_use: int):
        """A, B (P, n_use) in binary128 rounded to FP64 (compute_exact_mpfr_AB restated)."""
        vi = np.ascontiguousarray(cands.v_int, dtype=np.uint64)
        vf = np.ascontiguousarray(cands.v_frac, dtype=np.uint64)
        d = getattr(cands, "delta", None)
        d = None if d is None else np.ascontiguousarray(d, dtype=np.float64)
        P = vi.shape[0]
        A = np.empty((P, n_use))
        B = np.empty((P, n_use))
        G3 = np.ascontiguousarray(table.G3, dtype=np.uint64)
        self.L.orc_exact_AB(P, _p(vi), _p(vf), None if d is None else _p(d), int(n_use), _p(G3),
                            _p(np.ascontiguousarray(table.c_re)), _p(np.ascontiguousarray(table.c_im)),
                            _p(A), _p(B))
        return A, B

    def abs_sum(self, table, k: float, n_use: int) -> float:
        return self.L.orc_abs_sum(int(n_use), _p(np.ascontiguousarray(table.G3)), _p(np.ascontiguousarray(table.c_re)),
                                  _p(np.ascontiguousarray(table.c_im)), float(k))

    def gamma_from_G(self, G3):
        G3 = np.ascontiguousarray(G3, dtype=np.uint64)
        g = np.empty(G3.shape[0])
        self.L.orc_gamma_from_G(G3.shape[0], _p(G3), _p(g))
        return g

    def ref_peak_AB(self, refc, reft, n=None, want_top=False):
        """Restated compute_peak_AB (single-threaded); refc/reft from reference_format()."""
        x_lo, x_hi, dy0 = refc
        n = reft["n"] if n is None else n
        P = x_lo.shape[0]
        A = np.empty((P, n)); B = np.empty((P, n))
        top = np.empty((P, n), dtype=np.uint64) if want_top else None
        self.L.orc_ref_peak_AB(P, _p(x_lo), _p(x_hi), _p(dy0), n, _p(reft["alpha"]), _p(reft["gamma"]),
                               _p(reft["ghi_lo"]), _p(reft["ghi_hi"]), _p(reft["glo_lo"]), _p(reft["glo_hi"]),
                               _p(reft["psi_lo"]), _p(reft["psi_hi"]), _p(A), _p(B),
                               _p(top) if want_top else None)
        return (A, B, top) if want_top else (A, B)

    def fast_screen(self, x_lo, x_hi, reft, two_astar):
        """Restated ZeroData::fast_screen (search/fast_mertens_enum.cpp:108-142) over leaves
        x = x_hi 2^64 + x_lo on the reference layout; returns the per-leaf pass flags."""
        x_lo = np.ascontiguousarray(x_lo, dtype=np.uint64)
        x_hi = np.ascontiguousarray(x_hi, dtype=np.uint64)
        ta = np.ascontiguousarray(two_astar[:128], dtype=np.float64)
        g = np.ascontiguousarray(reft["gamma"][:128], dtype=np.float64)
        out = np.zeros(x_lo.shape[0], dtype=np.uint8)
        self.L.orc_fast_screen(x_lo.shape[0], _p(x_lo), _p(x_hi), _p(reft["ghi_lo"]), _p(reft["ghi_hi"]),
                               _p(reft["glo_lo"]), _p(reft["glo_hi"]), _p(reft["psi_lo"]), _p(reft["psi_hi"]),
                               _p(ta), _p(g), _p(out))
        return out

    def ref_polish(self, A, B, gamma, w, half, steps):
        P, n = A.shape
        hu, hp, dp = np.empty(P), np.empty(P), np.empty(P)
        self.L.orc_ref_polish(P, n, _p(np.ascontiguousarray(A)), _p(np.ascontiguousarray(B)),
                              _p(np.ascontiguousarray(gamma[:n])), _p(np.ascontiguousarray(w[:n])),
                              float(half), int(steps), _p(hu), _p(hp), _p(dp))
        return hu, hp, dp


# ------------------------------------------------------------------ reference layout adapter

def _rint_shift(x: int, s: int) -> int:
    """round-half-even(x / 2^s) for integers."""
    q, r = x >> s, x & ((1 << s) - 1)
    half = 1 << (s - 1)
    if r > half or (r == half and (q & 1)):
        q += 1
    return q


def reference_format(table, n=None, exact_psi=True):
    """The table in the reference's zeros_600k.bin field set (planar arrays).

    ghi = G 2^146 mod 2^128 and glo = rint(G 2^98) (round half to even) are exact integer
    transforms of the 64.128 fixed-point G, done limb-wise in numpy.  psi is computed from
    the FP64 c at 256 bits with mpmath (exact_psi) or in FP64 (top 53 bits only)."""
    n = table.G3.shape[0] if n is None else n
    G3 = np.ascontiguousarray(table.G3[:n], dtype=np.uint64)
    gi, g1, g2 = G3[:, 0], G3[:, 1], G3[:, 2]
    u = np.uint64
    out = {}
    # G 2^146 mod 2^128 = (g1 2^64 + g2) 2^18 mod 2^128
    out["ghi_hi"] = (g1 << u(18)) | (g2 >> u(46))
    out["ghi_lo"] = g2 << u(18)
    # G 2^98 = Gfix / 2^30 with Gfix = gi 2^128 + g1 2^64 + g2, rounded half to even
    hi = (gi << u(34)) | (g1 >> u(30))
    lo = (g1 << u(34)) | (g2 >> u(30))
    rem = g2 & u((1 << 30) - 1)
    half = u(1 << 29)
    up = (rem > half) | ((rem == half) & ((lo & u(1)) == u(1)))
    lo2 = lo + up.astype(np.uint64)
    hi = hi + ((lo2 < lo) & up).astype(np.uint64)
    out["glo_hi"], out["glo_lo"] = hi, lo2
    if exact_psi:
        import mpmath as mp
        out["psi_lo"] = np.empty(n, dtype=np.uint64)
        out["psi_hi"] = np.empty(n, dtype=np.uint64)
        with mp.workprec(256):
            two_pi = 2 * mp.pi
            for j in range(n):
                a = mp.atan2(mp.mpf(float(table.c_im[j])), mp.mpf(float(table.c_re[j])))
                psi = int(mp.nint(((-a / two_pi) % 1) * mp.mpf(2) ** 128)) & MASK128
                out["psi_lo"][j], out["psi_hi"][j] = psi & MASK64, psi >> 64
    else:
        f = np.mod(-np.arctan2(table.c_im[:n], table.c_re[:n]) / (2 * np.pi), 1.0)
        s = np.minimum(f * 2.0**64, np.nextafter(2.0**64, 0))
        out["psi_hi"] = s.astype(np.uint64)
        out["psi_lo"] = np.zeros(n, dtype=np.uint64)
    for key in ("ghi_lo", "ghi_hi", "glo_lo", "glo_hi", "psi_lo", "psi_hi"):
        out[key] = np.ascontiguousarray(out[key])
    out["alpha"] = np.ascontiguousarray(np.hypot(table.c_re[:n], table.c_im[:n]))
    out["gamma"] = np.ascontiguousarray(table.gamma[:n])
    out["n"] = n
    return out


def reference_candidates(cands):
    """x = floor(v 2^30) (u128 as lo/hi words) and dy0 = v - x 2^-30 (+ delta), in FP64."""
    P = cands.v_int.shape[0]
    x_lo = np.empty(P, dtype=np.uint64); x_hi = np.empty(P, dtype=np.uint64); dy0 = np.empty(P)
    for p in range(P):
        vi, vf = int(cands.v_int[p]), int(cands.v_frac[p])
        x = (vi << 30) | (vf >> 34)
        x_lo[p], x_hi[p] = x & MASK64, x >> 64
        dy0[p] = float(vf & ((1 << 34) - 1)) * 2.0**-64 + float(cands.delta[p])
    return x_lo, x_hi, dy0


# ------------------------------------------------------------------ ZeroData::polish restated

def zerodata_polish(top, two_astar, gamma, thresholds=(0.895, 0.918, 0.948)):
    """search/gpu_mertens_stream.cu:381-505 for one hit, in FP64 numpy: top = the signed top word
    of ph = xh ghi + xl glo - psi (int64 per zero), angle = top pi/2^63; five grid stages with
    early exits.  Returns (best_h, best_dy)."""
    SCALE = np.pi / 9223372036854775808.0
    ang = top.astype(np.float64) * SCALE
    g = np.asarray(gamma, np.float64)
    ta = np.asarray(two_astar, np.float64)
    n = len(g)

    def grid(K, m_half, step, centre, base_ang):
        dys = centre + np.arange(-m_half, m_half + 1) * step
        A = ta[:K] * np.cos(base_ang[:K])
        B = ta[:K] * np.sin(base_ang[:K])
        th = g[None, :K] * (dys - centre)[:, None]
        s = (A[None, :] * np.cos(th) - B[None, :] * np.sin(th)).sum(axis=1)
        j = int(np.argmax(np.abs(s)))
        return float(s[j]), float(dys[j]), float(abs(s[j]))

    best_h, best_dy, b = grid(256, 38, 1.5e-4, 0.0, ang)
    if thresholds[0] is not None and b < thresholds[0]:
        return best_h, best_dy
    best_h, best_dy, b = grid(512, 228, 2.5e-5, 0.0, ang)
    if thresholds[1] is not None and b < thresholds[1]:
        return best_h, best_dy
    centre = best_dy
    best_h, best_dy, b = grid(2048, 60, 1e-5, centre, ang + g * centre)
    if thresholds[2] is not None and b < thresholds[2]:
        return best_h, best_dy
    centre = best_dy
    K2 = min(15000, n)
    dys = centre + np.arange(-320, 321) * 2.5e-6
    s = np.array([(ta[:K2] * np.cos(ang[:K2] + g[:K2] * dy)).sum() for dy in dys])
    best_dy = float(dys[int(np.argmax(np.abs(s)))])
    centre = best_dy
    dys = centre + np.arange(-120, 121) * 5e-7
    s = np.array([(ta * np.cos(ang + g * dy)).sum() for dy in dys])
    j = int(np.argmax(np.abs(s)))
    return float(s[j]), float(dys[j])


# ------------------------------------------------------------------ reference evaluator

class RefLib:
    """The reference's compiled evaluator (compute_peak_AB, polish_peaks_with_weights)."""

    def __init__(self):
        if not os.path.exists(REF_SO):
            build()
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        L = C.CDLL(REF_SO)
        L.compute_peak_AB.argtypes = [C.c_int] + [C.c_void_p] * 3 + [C.c_int] + [C.c_void_p] * 10
        L.compute_peak_AB.restype = None
        L.polish_peaks_with_weights.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 4 + [C.c_double, C.c_int] + [C.c_void_p] * 3
        L.polish_peaks_with_weights.restype = None
        self.L = L

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO)

    def peak_AB(self, refc, reft, n=None):
        x_lo, x_hi, dy0 = refc
        n = reft["n"] if n is None else n
        P = x_lo.shape[0]
        A = np.empty((P, n)); B = np.empty((P, n))
        self.L.compute_peak_AB(P, _p(x_lo), _p(x_hi), _p(dy0), n, _p(reft["alpha"]), _p(reft["gamma"]),
                               _p(reft["ghi_lo"]), _p(reft["ghi_hi"]), _p(reft["glo_lo"]), _p(reft["glo_hi"]),
                               _p(reft["psi_lo"]), _p(reft["psi_hi"]), _p(A), _p(B))
        return A, B

    def polish(self, A, B, gamma, w, half, steps):
        P, n = A.shape
        hu, hp, dp = np.empty(P), np.empty(P), np.empty(P)
        self.L.polish_peaks_with_weights(P, n, _p(np.ascontiguousarray(A)), _p(np.ascontiguousarray(B)),
                                         _p(np.ascontiguousarray(gamma[:n])), _p(np.ascontiguousarray(w[:n])),
                                         float(half), int(steps), _p(hu), _p(hp), _p(dp))
        return hu, hp, dp


# ------------------------------------------------------------------ the reference's ZeroData

class ZeroDataRef:
    """The reference enumerator's ZeroData (search/fast_mertens_enum.cpp:27-277), compiled from its
    source by the Makefile, on a zeros.bin file (at least 15,000 zeros: polish() reads that many).
    Leaves and hits are x = floor(y 2^30) as u128 (x_lo, x_hi words), as the enumerators hold them."""

    def __init__(self, zeros_bin_path: str):
        if not os.path.exists(ZD_SO):
            build()
        if not os.path.exists(ZD_SO):
            raise FileNotFoundError(ZD_SO)
        L = C.CDLL(ZD_SO)
        L.zd_load.argtypes = [C.c_char_p]
        L.zd_load.restype = C.c_void_p
        L.zd_free.argtypes = [C.c_void_p]
        L.zd_n_zeros.argtypes = [C.c_void_p]
        L.zd_fast_screen.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
        L.zd_polish.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        self.L = L
        self.h = L.zd_load(zeros_bin_path.encode())
        if not self.h:
            raise OSError(f"ZeroData::load failed on {zeros_bin_path}")
        if L.zd_n_zeros(self.h) < 15000:
            self.close()
            raise ValueError("ZeroData::polish needs at least 15,000 zeros")

    @staticmethod
    def available() -> bool:
        return os.path.exists(ZD_SO)

    def fast_screen(self, x_lo, x_hi):
        x_lo = np.ascontiguousarray(x_lo, dtype=np.uint64)
        x_hi = np.ascontiguousarray(x_hi, dtype=np.uint64)
        out = np.zeros(x_lo.shape[0], dtype=np.uint8)
        self.L.zd_fast_screen(self.h, x_lo.shape[0], _p(x_lo), _p(x_hi), _p(out))
        return out

    def polish(self, x_lo, x_hi):
        x_lo = np.ascontiguousarray(x_lo, dtype=np.uint64)
        x_hi = np.ascontiguousarray(x_hi, dtype=np.uint64)
        h, dy = np.empty(x_lo.shape[0]), np.empty(x_lo.shape[0])
        self.L.zd_polish(self.h, x_lo.shape[0], _p(x_lo), _p(x_hi), _p(h), _p(dy))
        return h, dy

    def close(self):
        if getattr(self, "h", None):
            self.L.zd_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
