"""Candidate scoring under the search drivers' weight kernels, on the GPU without A/B matrices.

search/eval_tech1_600k.py:216-273 (and eval_tech2_hdrop_600k.py, eval_sub35_candidates.py) score
their candidates by compute_peak_AB over all N zeros followed by one polish_peaks_with_weights per
weight vector (grid_half_width 2.5e-4, 40 steps): the P x N A/B matrices are built once and read
five times.  Here each weight vector is registered with the table once and all polishes are one
mb_polish_peaks_weights call, which writes the exact-phase (A_j, B_j) of the candidates to device
memory once and runs every weight's polish from it:

    table = k2.ZeroTable.from_data(data)
    slots = register(table, reference_weights(data.gamma))   # once per table
    cands = candidates_from_x(x, dy)                 # the drivers' x = floor(y 2^30) and dy
    res = score(table, cands, slots)
    h_unpol, h_pol, ddy_pol = res["jp"]
"""
from __future__ import annotations

import numpy as np

from . import path1, synth

MASK30 = (1 << 30) - 1


def reference_weights(gamma: np.ndarray) -> dict[str, np.ndarray]:
    """The five weight vectors of search/eval_tech1_600k.py:243-249 over the table's zeros:
    Jurkat-Peyerimhoff (u = gamma / gamma_max), Gaussians exp(-1.5e-10 gamma^2) and
    exp(-1e-10 gamma^2), raw (1) and the first 10,000 zeros only."""
    g = np.ascontiguousarray(gamma, dtype=np.float64)
    u = g / g[-1]
    first = np.zeros_like(g)
    first[:10_000] = 1.0
    return {"jp": (1.0 - u) * np.cos(np.pi * u) + np.sin(np.pi * u) / np.pi,
            "g15": np.exp(-1.5e-10 * g * g),
            "g10": np.exp(-1.0e-10 * g * g),
            "raw": np.ones_like(g),
            "10k": first}


def candidates_from_x(x, dy=None) -> synth.Candidates:
    """Candidates from the drivers' x = floor(y 2^30) (u128, Python ints) and FP64 offsets dy:
    v = x 2^-30 exactly in 64.64 fixed point, delta = dy."""
    xs = [int(a) for a in x]
    vi = np.array([a >> 30 for a in xs], dtype=np.uint64)
    vf = np.array([(a & MASK30) << 34 for a in xs], dtype=np.uint64)
    d = np.zeros(len(xs)) if dy is None else np.ascontiguousarray(dy, dtype=np.float64)
    if d.shape != (len(xs),):
        raise ValueError("dy must have one offset per candidate")
    return synth.Candidates(vi, vf, d.copy())


def register(table, weights: dict[str, np.ndarray]) -> dict[str, int]:
    """name -> slot of each weight vector (length table.n) registered with the table; a driver
    registers its vectors once and passes the slots to every score() call."""
    return {name: table.add_weights(w) for name, w in weights.items()}


def score(table, cands, weights: dict, grid_half_width: float = 2.5e-4, grid_steps: int = 40,
          n_zeros: int | None = None) -> dict[str, tuple[np.ndarray, np.ndarray, np.ndarray]]:
    """name -> (h_unpol, h_pol, ddy_pol) of polish_peaks_with_weights for each weight vector, over
    the first n_zeros zeros (all by default).  Each value of `weights` is a slot from register()
    (or ZeroTable.add_weights), or a weight vector of length table.n, which is registered first
    (hashing it to find a slot registered before: milliseconds per vector, so pass slots in a
    loop)."""
    names = list(weights)
    slots = [w if isinstance(w, (int, np.integer)) else table.add_weights(w) for w in weights.values()]
    hu, hp, dp = path1.polish_peaks_weights(table, cands, slots, n_zeros, grid_half_width, grid_steps)
    return {name: (hu[i], hp[i], dp[i]) for i, name in enumerate(names)}
