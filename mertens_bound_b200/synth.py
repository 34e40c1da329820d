"""Seeded synthetic zero tables and candidate points for the K2 evaluator.

The real zeta zeros (Odlyzko's tables, the Arb zero cache) are not part of this
repository.  The generator reproduces their statistics closely enough to exercise
every code path at the real sizes:

* gamma_j solves N(gamma) = j - 1/2 + u_j with N(T) = (T/2pi) log(T/(2pi e)) + 7/8
  and u_j ~ U(-0.3, 0.3), so the zeros are strictly increasing with the
  Riemann-von Mangoldt density.
* G_j = gamma_j / 2pi is stored as unsigned 64.128 fixed point (three u64 limbs
  [int, hi, lo]): the binary expansion of the FP64 quotient followed by uniformly
  random bits below its last bit.  The stored G is the truth; the FP64 gamma_j
  handed to the evaluator is 2pi G_j rounded to double (80-bit extended product,
  so |gamma_f64 - 2pi G| <= 1 ulp).
* c_j = 1/(rho_j zeta'_j) with rho_j = 1/2 + i gamma_j and
  zeta'_j = exp(X_j) e^{i theta_j}, X_j ~ N(log log(gamma_j/2pi), 1/2 log log(gamma_j/2pi))
  (second argument is the variance, clamped at 0.01 for the lowest zeros),
  theta_j ~ U[0, 2pi).  c_j is stored as an FP64 pair and is exact by definition.
* Candidates v = v_int + v_frac 2^-64 with v_int ~ U[3.4e18, 3.6e18] and a uniform
  64-bit fraction.

The reference's Peak2 point (certification/certify_K2.py:41,
v = 3484971332733132396.5383341489440461) is provided as PEAK2.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from fractions import Fraction

import numpy as np

TWO_PI = 2.0 * math.pi
_MASK64 = (1 << 64) - 1

PEAK2_STR = "3484971332733132396.5383341489440461"


def zero_count(T):
    """Smooth zero count N(T) = (T/2pi) log(T/(2pi e)) + 7/8."""
    T = np.asarray(T, dtype=np.float64)
    return T / TWO_PI * np.log(T / (TWO_PI * math.e)) + 0.875


def _solve_gamma(y: np.ndarray) -> np.ndarray:
    """Solve N(T) = y for T > 2pi (Lambert-W start, three Newton steps)."""
    from scipy.special import lambertw

    z = (y - 0.875) / math.e
    x = np.exp(lambertw(z, 0).real)
    T = TWO_PI * math.e * x
    for _ in range(3):
        T = T - (zero_count(T) - y) / (np.log(T / TWO_PI) / TWO_PI)
    return T


def fixed_from_double(g: np.ndarray, rng: np.random.Generator | None) -> np.ndarray:
    """Exact 64.128 fixed point of positive doubles g (2 <= g < 2^32), with uniformly
    random bits filled in below each double's last mantissa bit when rng is given."""
    m, e = np.frexp(g)                      # g = m 2^e, 0.5 <= m < 1
    M = (m * 2.0**53).astype(np.uint64)     # exact 53-bit integer mantissa
    s = (e.astype(np.int64) - 53 + 64)      # g 2^64 = M << s ; s in [13, 43] for g in [2, 2^32)
    if np.any(s < 1) or np.any(s > 63):
        raise ValueError("fixed_from_double expects 2 <= g < 2^32")
    s = s.astype(np.uint64)
    hi = np.left_shift(M, s)                # low 64 bits of M << s  (fraction limb 1)
    gi = np.right_shift(M, np.uint64(64) - s)
    lo = np.zeros_like(hi)
    if rng is not None:
        r_hi = rng.integers(0, _MASK64, size=g.shape, dtype=np.uint64, endpoint=True)
        r_lo = rng.integers(0, _MASK64, size=g.shape, dtype=np.uint64, endpoint=True)
        mask = np.left_shift(np.uint64(1), s) - np.uint64(1)
        hi = hi | (r_hi & mask)
        lo = r_lo
    return np.stack([gi, hi, lo], axis=1)


_TWO_PI_LD = np.longdouble("6.28318530717958647692528676655900576839")


def gamma_from_fixed(G3: np.ndarray) -> np.ndarray:
    """FP64 gamma = 2pi G from the 64.128 limbs (x87 extended product, one rounding)."""
    G = (G3[:, 0].astype(np.longdouble) + np.ldexp(G3[:, 1].astype(np.longdouble), -64)
         + np.ldexp(G3[:, 2].astype(np.longdouble), -128))
    return (G * _TWO_PI_LD).astype(np.float64)


@dataclass
class ZeroTableData:
    """Host-side synthetic table: G3 (N,3) uint64, gamma/c_re/c_im (N,) float64."""
    G3: np.ndarray
    gamma: np.ndarray
    c_re: np.ndarray
    c_im: np.ndarray
    seed: int

    @property
    def n(self) -> int:
        return int(self.gamma.shape[0])

    def truncate(self, n: int) -> "ZeroTableData":
        return ZeroTableData(self.G3[:n].copy(), self.gamma[:n].copy(), self.c_re[:n].copy(),
                             self.c_im[:n].copy(), self.seed)

    def count_below(self, T: float) -> int:
        """Number of zeros with gamma < T (the table is sorted)."""
        if not math.isfinite(T):
            return self.n
        return int(np.searchsorted(self.gamma, T, side="left"))


def make_table(n: int, seed: int = 1) -> ZeroTableData:
    """The first n synthetic zeros (j = 1..n) for a given seed."""
    ss = np.random.SeedSequence([seed, 0x4B32])
    r_u, r_bits, r_x, r_th = (np.random.default_rng(s) for s in ss.spawn(4))
    j = np.arange(1, n + 1, dtype=np.float64)
    y = j - 0.5 + r_u.uniform(-0.3, 0.3, n)
    gam0 = _solve_gamma(y)
    G3 = fixed_from_double(gam0 / TWO_PI, r_bits)
    gamma = gamma_from_fixed(G3)
    if n > 1 and not np.all(np.diff(gamma) > 0):
        raise RuntimeError("synthetic zeros are not strictly increasing")
    ll = np.log(np.log(gamma / TWO_PI))
    X = r_x.normal(ll, np.sqrt(np.maximum(0.5 * ll, 0.01)))
    th = r_th.uniform(0.0, TWO_PI, n)
    zp = np.exp(X) * np.exp(1j * th)
    rho = 0.5 + 1j * gamma
    c = 1.0 / (rho * zp)
    return ZeroTableData(G3=np.ascontiguousarray(G3), gamma=gamma, c_re=np.ascontiguousarray(c.real),
                         c_im=np.ascontiguousarray(c.imag), seed=seed)


def make_table_below(T0: float, seed: int = 1) -> ZeroTableData:
    """All synthetic zeros with gamma < T0."""
    n_max = int(math.ceil(float(zero_count(T0)))) + 2
    t = make_table(n_max, seed)
    return t.truncate(t.count_below(T0))


@dataclass
class Candidates:
    """Candidate points v = v_int + v_frac 2^-64 + delta."""
    v_int: np.ndarray
    v_frac: np.ndarray
    delta: np.ndarray

    @property
    def n(self) -> int:
        return int(self.v_int.shape[0])

    def subset(self, idx) -> "Candidates":
        return Candidates(self.v_int[idx].copy(), self.v_frac[idx].copy(), self.delta[idx].copy())


def make_candidates(P: int, seed: int = 2) -> Candidates:
    rng = np.random.default_rng(np.random.SeedSequence([seed, 0x5643]))
    v_int = rng.integers(3_400_000_000_000_000_000, 3_600_000_000_000_000_000, size=P,
                         dtype=np.uint64, endpoint=True)
    v_frac = rng.integers(0, _MASK64, size=P, dtype=np.uint64, endpoint=True)
    return Candidates(v_int, v_frac, np.zeros(P, dtype=np.float64))


def fixed_from_decimal(s: str) -> tuple[int, int]:
    """(v_int, v_frac) = (floor(v), floor(frac(v) 2^64)) of a decimal string."""
    f = Fraction(s)
    vi = int(f)
    vf = int((f - vi) * (1 << 64))
    return vi, vf


def peak2_candidate() -> Candidates:
    vi, vf = fixed_from_decimal(PEAK2_STR)
    return Candidates(np.array([vi], dtype=np.uint64), np.array([vf], dtype=np.uint64),
                      np.zeros(1, dtype=np.float64))


def batched_uneven_groups():
    """The batched workload: 12 groups of unequal size (64..4096, 16,384 candidates in all), one
    per (T, k) in {1e5, 3e5, 6e5, 1.3e6} x {3e-9, 1e-9, 1.5e-10}.  Returns (counts, ks, Ts)."""
    counts = [4096, 64, 2048, 256, 3072, 128, 1536, 512, 1024, 2048, 1024, 576]
    Ts = [T for T in (1e5, 3e5, 6e5, 1.3e6) for _ in range(3)]
    ks = [k for _ in range(4) for k in (3e-9, 1e-9, 1.5e-10)]
    assert sum(counts) == 16_384 and min(counts) >= 64 and max(counts) <= 4096
    return counts, ks, Ts


# The enumerators' screen and hit polish compare absolute scores with fixed thresholds (0.81 ..
# 0.948).  With the generator's coefficients the first 64 zeros carry sum 2|c| w = 1.08, so random
# leaves never reach them (the enumerators' leaves come from a lattice search that aligns the
# phases); a table with c scaled by 3 lets about 9% of random leaves pass the screen and run the
# polish to its last stage, so both sides of every threshold are exercised.
ENUM_C_SCALE = 3.0


def enumerator_table(n: int = 40_000, seed: int = 1, c_scale: float = ENUM_C_SCALE) -> ZeroTableData:
    """make_table(n, seed) with every coefficient c multiplied by c_scale."""
    t = make_table(n, seed=seed)
    return ZeroTableData(t.G3, t.gamma, t.c_re * c_scale, t.c_im * c_scale, t.seed)


def leaves_x(count: int, seed: int) -> list:
    """x = floor(v 2^30) (Python ints, the enumerators' u128 leaf form) of make_candidates(count, seed)."""
    c = make_candidates(count, seed=seed)
    return [(int(a) << 30) | (int(b) >> 34) for a, b in zip(c.v_int, c.v_frac)]


# The five workloads (sizes, cutoffs and Gaussian widths) the evaluator is measured on.
WORKLOADS = {
    "small_plain": dict(n_zeros=10_000, T=math.inf, k=3e-9, P=64, table_seed=1, cand_seed=2),
    "search_scoring": dict(T0=3e5, T=3e5, k=3e-9, P=4096, table_seed=1, cand_seed=3),
    "certified_full": dict(n_zeros=2_325_572, T=1.3e6, k=1.5e-10, P=1, table_seed=1),
    "batched_uneven": dict(n_zeros=2_325_572, P=16_384, groups=12, table_seed=1, cand_seed=4),
    "newton_polish": dict(n_zeros=2_325_572, T=1.3e6, k=1.5e-10, P=1024, table_seed=1, cand_seed=5),
}
