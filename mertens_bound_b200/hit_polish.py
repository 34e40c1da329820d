"""Hit polish of the lattice enumerators on the GPU (row "enumerator scoring").

search/gpu_mertens_stream.cu:381-505 (ZeroData::polish; the same 5 stages in
search/fast_mertens_enum.cpp:145-276) refines every enumeration hit on the CPU with a cascade of
FP64 grid scans of h(y) = sum_j two_astar_j cos(theta_j + gamma_j dy), two_astar_j =
2|c_j| exp(-3e-9 gamma_j^2), stopping early when the best |h| stays below a threshold:

  stage  zeros   grid points           step     centre           exit if best |h| <
  0      256     m in [-38, 38]        1.5e-4   0                0.895
  1      512     m in [-228, 228]      2.5e-5   0                0.918 (enum: 0.915)
  2      2048    m in [-60, 60]        1e-5     stage-1 best     0.948 (enum: 0.945)
  3      15000   m in [-320, 320]      2.5e-6   stage-2 best     (moves the centre only)
  4      all     m in [-120, 120]      5e-7     stage-3 best     returns (h, dy)

Here each stage is one mb_hit_scan call over all hits still alive (one CTA per hit), with
exact phases at every grid point; hits are x = floor(y 2^30) as in the reference
(gpu_mertens_stream.cu:711) or 64.64 points.
"""
from __future__ import annotations

from dataclasses import dataclass
from fractions import Fraction

import numpy as np

from . import k2
from ._lib import check, lib, ptr

MASK64 = (1 << 64) - 1
STAGES = (  # (zeros, m_half, step, centre from previous stage, exit threshold)
    (256, 38, 1.5e-4, False, 0.895),
    (512, 228, 2.5e-5, False, 0.918),
    (2048, 60, 1e-5, True, 0.948),
    (15000, 320, 2.5e-6, True, None),
    (None, 120, 5e-7, True, None),
)
ENUM_THRESHOLDS = (0.895, 0.915, 0.945)      # fast_mertens_enum.cpp:177,203,236


@dataclass
class HitResult:
    h: np.ndarray          # best h per hit
    dy: np.ndarray         # offset of the best point from the hit (FP64)
    stage: np.ndarray      # last stage run per hit (0..4)


def _fixed(step: float) -> int:
    """64.64 fixed point of a positive double (exact for the stage steps' binary values)."""
    q = Fraction(step)
    return int(q * (1 << 64))


def points_from_x(x) -> np.ndarray:
    """(n, 2) u64 (v_int, v_frac) of hits x = floor(y 2^30) (u128 as Python ints)."""
    out = np.empty((len(x), 2), dtype=np.uint64)
    for i, xi in enumerate(x):
        xi = int(xi)
        out[i, 0] = xi >> 30
        out[i, 1] = (xi & ((1 << 30) - 1)) << 34
    return out


def _scan(table, pts_fixed, k, n_use, step_fixed, m_half):
    P = len(pts_fixed)
    vi = np.array([p >> 64 for p in pts_fixed], dtype=np.uint64)
    vf = np.array([p & MASK64 for p in pts_fixed], dtype=np.uint64)
    n_m = 2 * m_half + 1
    h = np.empty((P, n_m))
    check(lib().mb_hit_scan(table.handle, P, ptr(vi), ptr(vf), float(k), int(n_use), step_fixed >> 64,
                            step_fixed & MASK64, -m_half, n_m, ptr(h)))
    return h


def polish_hits(table: k2.ZeroTable, points: np.ndarray, k: float = 3e-9, thresholds=None) -> HitResult:
    """Run the staged polish for every hit (points: (n, 2) u64 v_int, v_frac)."""
    thr = [s[4] for s in STAGES[:3]] if thresholds is None else list(thresholds)
    n = len(points)
    base = [(int(points[i, 0]) << 64) | int(points[i, 1]) for i in range(n)]
    centre = [0] * n                       # fixed-point offset of the current centre
    best_h = np.zeros(n)
    best_dy = np.zeros(n)
    stage = np.zeros(n, dtype=np.int64)
    alive = np.arange(n)
    for s, (K, m_half, step, recentre, _) in enumerate(STAGES):
        if len(alive) == 0:
            break
        n_use = table.n if K is None else min(K, table.n)
        sf = _fixed(step)
        pts = [(base[i] + (centre[i] if recentre else 0)) & ((1 << 128) - 1) for i in alive]
        h = _scan(table, pts, k, n_use, sf, m_half)
        j = np.argmax(np.abs(h), axis=1)                       # first maximum, like the reference
        hb = h[np.arange(len(alive)), j]
        for idx, i in enumerate(alive):
            off = (int(j[idx]) - m_half) * sf
            c = (centre[i] if recentre else 0) + off
            stage[i] = s
            if s != 3:                                         # stage 3 only moves the centre
                best_h[i] = hb[idx]
            centre[i] = c
            best_dy[i] = float(Fraction(c, 1 << 64))
        if s < 3 and thr[s] is not None:
            keep = np.abs(hb) >= thr[s]
            alive = alive[keep]
    return HitResult(best_h, best_dy, stage)


# Leaf screens: (zeros at the end of each stage, thresholds) of the reference's proxies.
SCREEN_GPU = ((64, 128, 256), (0.78, 0.855, 0.892))     # gpu_mertens_stream.cu:203-250
SCREEN_CPU = ((64, 128), (0.810, 0.875))                # fast_mertens_enum.cpp:108-142
SCREEN_STEP = 0.0014                                    # offset between the 7 proxy points


@dataclass
class ScreenResult:
    hits: np.ndarray         # indices of the leaves that passed every stage, ascending
    hit_scores: np.ndarray   # (n_hits, n_stages) max_m |S_m| after each stage
    scores: np.ndarray | None  # (P, n_stages) for every leaf (-1 where a stage was not reached)


def screen_leaves(table: k2.ZeroTable, points: np.ndarray, k: float = 3e-9, stages=SCREEN_GPU,
                  step: float = SCREEN_STEP, max_hits: int | None = None, all_scores: bool = False) -> ScreenResult:
    """The enumerators' staged leaf screen (search/fast_mertens_enum.cpp:108-142,
    search/gpu_mertens_stream.cu:192-250) on 64.64 points (n, 2): per leaf the sums
    S_m = sum_j 2|c_j| exp(-k gamma_j^2) cos(gamma_j (y + m step) + arg c_j), m = -3..3, over the
    zeros of each stage; a leaf survives a stage if max_m |S_m| >= that stage's threshold."""
    ends, thr = stages
    ends = np.ascontiguousarray(ends, dtype=np.int64)
    thr = np.ascontiguousarray(thr, dtype=np.float32)
    if ends.shape != thr.shape or ends.ndim != 1:
        raise ValueError("stage ends and thresholds must be 1-D of equal length")
    pts = np.ascontiguousarray(points, dtype=np.uint64)
    vi, vf = np.ascontiguousarray(pts[:, 0]), np.ascontiguousarray(pts[:, 1])
    P, S = vi.shape[0], ends.shape[0]
    cap = P if max_hits is None else int(max_hits)
    hits = np.empty(max(cap, 0), dtype=np.int64)
    hsc = np.empty((max(cap, 0), S), dtype=np.float32)
    sc = np.empty((P, S), dtype=np.float32) if all_scores else None
    n = np.zeros(1, dtype=np.int64)
    st = _fixed(step)
    check(lib().mb_screen(table.handle, P, ptr(vi), ptr(vf), float(k), st >> 64, st & MASK64, S, ptr(ends),
                          ptr(thr), cap, ptr(hits), ptr(hsc), ptr(n), ptr(sc)))
    m = int(n[0])
    return ScreenResult(hits[:m].copy(), hsc[:m].copy(), sc)


def screen_leaves_dev(table: k2.ZeroTable, d_v_int: int, d_v_frac: int, P: int, d_hits: int, d_hit_scores: int,
                      d_n_hits: int, max_hits: int, k: float = 3e-9, stages=SCREEN_GPU, step: float = SCREEN_STEP,
                      d_scores: int = 0, stream: int = 0) -> None:
    """screen_leaves on device arrays (pointers as ints: P u64 v_int and v_frac leaves; max_hits
    int64 hit slots, max_hits x n_stages float32 hit scores, one u64 hit count; optional P x
    n_stages float32 scores), asynchronous on `stream`; the hits come in arbitrary order."""
    ends, thr = stages
    ends = np.ascontiguousarray(ends, dtype=np.int64)
    thr = np.ascontiguousarray(thr, dtype=np.float32)
    if ends.shape != thr.shape or ends.ndim != 1:
        raise ValueError("stage ends and thresholds must be 1-D of equal length")
    st = _fixed(step)
    check(lib().mb_screen_dev(table.handle, int(P), d_v_int, d_v_frac, float(k), st >> 64, st & MASK64,
                              ends.shape[0], ptr(ends), ptr(thr), int(max_hits), d_hits, d_hit_scores, d_n_hits,
                              d_scores or None, stream))
