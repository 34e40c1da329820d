"""The tier kernels' phase arithmetic, emulated operation by operation with exact rounding, against
the exact phase frac(v G + psi) (Python integers and Fractions).

* light tier, light_phase32_fused (csrc/k2_light.cuh): 2 IMAD.lo + 3 DFMA on 1.5 2^52; the 32-bit
  phase word is within 2.4 units of 2^-32 turn (psi32 carries the +1 centring) for every zero
  with gamma < 3.29e6 (G's integer part below 2^19);
* heavy tier, heavy_tile (csrc/k2_fast.cu): the whole 2^-32-turn units in IMAD.lo, the FP64
  sums in two chains (one on 1.5 2^35), the FP32 low products, then the table index and the
  remainder from the bits of the FP64 sum plus the whole units times 2^17 (one 64-bit
  multiply-add); q/2048 + r is within 2^-48 turn of the exact phase for any 64.64 v and 32.128 G;
* plain kernel, sincos_phase64_tab (csrc/k2_plain.cu): cos/sin of the exact 64-bit phase word
  from a 2048-entry table and the exact remainder, within 2.5e-16 of mpmath's values.

The phase being reduced is search/path1_eval_fast.cpp:35-46's exact reduction of v gamma / 2pi.
"""
import random
import struct
from fractions import Fraction as Fr

import numpy as np

M32 = (1 << 32) - 1
MAGIC52 = 6755399441055744.0       # 1.5 2^52
MAGIC35 = 51539607552.0            # 1.5 2^35


def fma(a, b, c):
    """Round-to-nearest-even double of a b + c, computed exactly."""
    return float(Fr(a) * Fr(b) + Fr(c))


def f32(x):
    return float(np.float32(float(x)))


def fmaf(a, b, c):
    return f32(Fr(a) * Fr(b) + Fr(c))


def bits(d):
    return struct.unpack("<Q", struct.pack("<d", d))[0]


def from_bits(u):
    return struct.unpack("<d", struct.pack("<Q", u))[0]


def exact_phase(vi, vf, G, ps):
    return (Fr(vi) + Fr(vf, 1 << 64)) * Fr(G, 1 << 128) + Fr(ps, 1 << 64)


def turn_distance(x, y):
    e = (x - y) % 1
    return min(e, 1 - e)


def limbs(vi, vf, G):
    return (vi >> 32, vi & M32, vf >> 32, vf & M32,
            (G >> 128) & M32, (G >> 96) & M32, (G >> 64) & M32, (G >> 32) & M32, G & M32)


def light_fused_word(vi, vf, G, ps):
    a1, a0, d1, d0, gi, b1, b0, c1, _ = limbs(vi, vf, G)
    psi32 = (((ps + (1 << 31)) >> 32) + 1) & M32
    A0, A1 = float(a0), float(a1)
    VF = float(np.float64(float(Fr(vf)))) * 2.0 ** -64          # __ull2double_rn(v_frac) 2^-64
    b0s, c1s = b0 * 2.0 ** -32, c1 * 2.0 ** -32
    gh = float(gi * (1 << 32) + b1)                             # exact below 2^51
    lo32 = (a1 * b0 + a0 * b1 + psi32) & M32
    R1 = fma(A0, b0s, fma(A1, c1s, MAGIC52))
    R2 = fma(VF, gh, MAGIC52)
    return (lo32 + (bits(R1) & M32) + (bits(R2) & M32)) & M32


def heavy_q_r(vi, vf, G, ps):
    a1, a0, d1, d0, gi, b1, b0, c1, c0 = limbs(vi, vf, G)
    b0s, c1s, gis, b1s = (x * 2.0 ** -32 for x in (b0, c1, gi, b1))
    c0f, c1f, b0f, b1f = (f32(x * 2.0 ** -64) for x in (c0, c1, b0, b1))
    psi_hi = ((ps >> 32) + (1 << 20)) & M32
    psi_lo = f32((ps & M32) * 2.0 ** -32)
    L = (a1 * b0 + a0 * b1 + d1 * gi + psi_hi) & M32
    low = fmaf(f32(a1), c0f, fmaf(f32(a0), c1f, fmaf(f32(d1), b0f, fmaf(f32(d0), b1f, psi_lo))))
    p1 = fma(float(a0), b0s, fma(float(a1), c1s, low))
    p2 = fma(float(d0), gis, fma(float(d1), b1s, MAGIC35))
    w = (L * 131072 + bits(float(Fr(p1) + Fr(p2)))) & ((1 << 64) - 1)
    wh = w >> 32
    rb = from_bits((((wh & 0x3F) | 0x43300000) << 32) | (w & M32))
    r = fma(rb, 1.7763568394002505e-15, -8.000244140625)
    return (wh >> 6) & 2047, r


def _cases(n, seed, gi_bits):
    rng = random.Random(seed)
    for i in range(n):
        mode = i % 3
        vi = rng.getrandbits(64) if mode == 0 else (rng.getrandbits(7) if mode == 1 else 3_500_000_000_000_000_000 + rng.getrandbits(56))
        vf = rng.getrandbits(64)
        G = (rng.getrandbits(gi_bits) << 128) | rng.getrandbits(128)
        yield vi, vf, G, rng.getrandbits(64)


def test_light_fused_phase_word_within_2_4_units():
    worst = 0
    for vi, vf, G, ps in _cases(1500, 11, 19):
        u = light_fused_word(vi, vf, G, ps)
        worst = max(worst, turn_distance(Fr(u, 1 << 32), exact_phase(vi, vf, G, ps)) * (1 << 32))
    assert worst <= 2.4, float(worst)


def test_heavy_index_and_remainder_within_2_pow_minus_48():
    worst = 0
    for vi, vf, G, ps in _cases(1500, 12, 32):
        q, r = heavy_q_r(vi, vf, G, ps)
        assert 0 <= q < 2048 and abs(r) <= 2.0 ** -12
        worst = max(worst, turn_distance(Fr(q, 2048) + Fr(r), exact_phase(vi, vf, G, ps)))
    assert worst <= Fr(1, 1 << 48), float(worst)


def test_heavy_remainder_edges():
    """Whole units at the table-cell edges (L + F just below and above a multiple of 2^21) and the
    largest limbs: the index wraps mod 2048 and r stays within half a cell."""
    for vi, vf, G in ((M32 << 32 | M32, (1 << 64) - 1, (1 << 160) - 1), (0, 0, 0), (1, 0, 1 << 117)):
        for ps in (0, (1 << 64) - 1, 1 << 63, (1 << 43) - 1, 1 << 43):
            q, r = heavy_q_r(vi, vf, G, ps)
            assert 0 <= q < 2048 and abs(r) <= 2.0 ** -12
            assert turn_distance(Fr(q, 2048) + Fr(r), exact_phase(vi, vf, G, ps)) <= Fr(1, 1 << 48)


def test_plain_table_sincos_within_2e_16():
    """k2_plain.cu sincos_phase64_tab on the exact 64-bit phase word: table index from the top
    11 bits (plus half a step), exact remainder, two short polynomials and the rotation."""
    import mpmath as mp
    mp.mp.prec = 120
    tab = [(float(mp.cos(2 * mp.pi * i / 2048)), float(mp.sin(2 * mp.pi * i / 2048))) for i in range(2048)]
    rng = random.Random(13)
    worst = 0.0
    for it in range(3000):
        if it % 4:
            hi = rng.getrandbits(64)
        else:                            # cell edges: remainder at 0 and at +-half a step
            hi = ((rng.getrandbits(11) << 53) + rng.choice([0, 1, (1 << 52) - 1, 1 << 52, (1 << 53) - 1])) % (1 << 64)
        h = (hi + (1 << 52)) % (1 << 64)
        q = h >> 53
        rh = ((h >> 32) & 0x1FFFFF) - (1 << 20)
        r = fma(float(rh), 2.0 ** -32, float(Fr(h & M32, 1 << 64)))
        assert abs(r) <= 2.0 ** -12
        u = r * r
        s = r * fma(u, -41.341702240399755, 6.283185307179586)
        cm1 = u * fma(u, 64.93939402266829, -19.739208802178716)
        tx, ty = tab[q]
        cs = fma(tx, cm1, fma(-ty, s, tx))
        sn = fma(ty, cm1, fma(tx, s, ty))
        th = 2 * mp.pi * mp.mpf(hi) / 2 ** 64
        worst = max(worst, float(abs(cs - mp.cos(th))), float(abs(sn - mp.sin(th))))
    assert worst <= 2.5e-16, worst
