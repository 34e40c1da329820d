"""Zero-table file formats of the reference, read and written here.

* zeros_600k.bin (legacy/superseded/certify_peak2_600k.py:119-143, read by
  search/eval_tech1_600k.py:38-50): u64 n | f64 gamma[n] | f64 alpha[n] | u64 x 6 per zero,
  interleaved (ghi_lo, ghi_hi, glo_lo, glo_hi, psi_lo, psi_hi).
* zeros.bin (search/path1_build_zeros_100k.py:34-47, read by search/gpu_mertens_stream.cu:298-323):
  i32 n | f64 two_astar[n] (= 2|c| exp(-3e-9 gamma^2)) | f64 gamma[n] | u64 planar ghi_lo, ghi_hi,
  glo_lo, glo_hi, psi_lo, psi_hi.
* zero cache text (certification/certify_K2.py:65-97): one line per zero,
  "gamma\\tRe c\\tIm c\\t|zeta'| lower" with Arb ball strings "[mid +/- rad]".

Field meanings (search/path1_build_zeros_100k.py:102-104): ghi = rint(G 2^146) mod 2^128,
glo = rint(G 2^98), psi = rint(((-arg c / 2pi) mod 1) 2^128), alpha = |c|, G = gamma/2pi.
ghi carries the bits of G from 2^-18 down to 2^-146 exactly; glo the integer part and the
bits down to 2^-98 (rounded), so the 64.128 fixed point G is recovered exactly from the pair.
"""
from __future__ import annotations

import math
import os
import re
import struct
from dataclasses import dataclass

import numpy as np

from .synth import ZeroTableData

u = np.uint64
_KEYS = ("ghi_lo", "ghi_hi", "glo_lo", "glo_hi", "psi_lo", "psi_hi")


class FormatError(ValueError):
    """A table file is truncated, inconsistent or malformed."""


# ------------------------------------------------------------------ fixed-point conversions

def G3_from_ghi_glo(ghi_lo, ghi_hi, glo_lo, glo_hi) -> np.ndarray:
    """Exact 64.128 fixed-point G (n x 3 u64) from the reference's (ghi, glo) pair."""
    ghi_lo, ghi_hi = np.asarray(ghi_lo, u), np.asarray(ghi_hi, u)
    glo_lo, glo_hi = np.asarray(glo_lo, u), np.asarray(glo_hi, u)
    if np.any(ghi_lo & u((1 << 18) - 1)):
        raise FormatError("ghi has nonzero bits below 2^-146 (not G 2^146 mod 2^128)")
    g_lo = (ghi_lo >> u(18)) | (ghi_hi << u(46))          # G 2^128 bits 0..63
    mid46 = ghi_hi >> u(18)                                # bits 64..109
    low30 = g_lo & u((1 << 30) - 1)                        # bits 0..29 (dropped by glo's rounding)
    bit30 = (g_lo >> u(30)) & u(1)
    half = u(1 << 29)
    up = ((low30 > half) | ((low30 == half) & (bit30 == u(1)))).astype(u)
    t_lo = glo_lo - up                                     # glo truncated instead of rounded
    t_hi = glo_hi - (glo_lo < up).astype(u)
    # consistency: truncated glo bits 0..79 must equal G 2^128 bits 30..109
    want_lo = (g_lo >> u(30)) | (mid46 << u(34))
    want_hi16 = (mid46 >> u(30)) & u(0xFFFF)
    if np.any(t_lo != want_lo) or np.any((t_hi & u(0xFFFF)) != want_hi16):
        raise FormatError("ghi and glo disagree (inconsistent table)")
    top18 = (t_hi >> u(16)) & u((1 << 18) - 1)             # bits 110..127
    g_int = t_hi >> u(34)                                  # bits 128..
    g_hi = (top18 << u(46)) | mid46
    return np.ascontiguousarray(np.stack([g_int, g_hi, g_lo], axis=1))


def ghi_glo_from_G3(G3):
    """(ghi_lo, ghi_hi, glo_lo, glo_hi) of a 64.128 fixed-point G (round half to even for glo)."""
    G3 = np.asarray(G3, u)
    gi, g1, g2 = G3[:, 0], G3[:, 1], G3[:, 2]
    ghi_hi = (g1 << u(18)) | (g2 >> u(46))
    ghi_lo = g2 << u(18)
    hi = (gi << u(34)) | (g1 >> u(30))
    lo = (g1 << u(34)) | (g2 >> u(30))
    rem = g2 & u((1 << 30) - 1)
    half = u(1 << 29)
    up = ((rem > half) | ((rem == half) & ((lo & u(1)) == u(1)))).astype(u)
    lo2 = lo + up
    hi = hi + ((lo2 < lo) & (up == u(1))).astype(u)
    return ghi_lo, ghi_hi, lo2, hi


def psi_from_c(c_re, c_im, exact: bool = True):
    """psi = rint(((-arg c / 2pi) mod 1) 2^128) as (lo, hi) u64 words."""
    n = len(c_re)
    lo, hi = np.zeros(n, u), np.zeros(n, u)
    if exact:
        import mpmath as mp
        with mp.workprec(256):
            two_pi = 2 * mp.pi
            for j in range(n):
                a = mp.atan2(mp.mpf(float(c_im[j])), mp.mpf(float(c_re[j])))
                v = int(mp.nint(((-a / two_pi) % 1) * mp.mpf(2) ** 128)) & ((1 << 128) - 1)
                lo[j], hi[j] = v & ((1 << 64) - 1), v >> 64
    else:
        f = np.mod(-np.arctan2(c_im, c_re) / (2 * np.pi), 1.0)
        hi = np.minimum(f * 2.0 ** 64, np.nextafter(2.0 ** 64, 0)).astype(u)
    return lo, hi


def c_from_alpha_psi(alpha, psi_lo, psi_hi):
    """c = alpha exp(-2 pi i psi 2^-128) in FP64."""
    turns = (np.asarray(psi_hi, u).astype(np.float64) + np.asarray(psi_lo, u).astype(np.float64) * 2.0 ** -64) * 2.0 ** -64
    ang = -2 * np.pi * turns
    a = np.asarray(alpha, np.float64)
    return a * np.cos(ang), a * np.sin(ang)


def reference_fields(table: ZeroTableData, exact_psi: bool = True) -> dict:
    ghi_lo, ghi_hi, glo_lo, glo_hi = ghi_glo_from_G3(table.G3)
    psi_lo, psi_hi = psi_from_c(table.c_re, table.c_im, exact=exact_psi)
    return dict(n=table.n, gamma=table.gamma.copy(), alpha=np.hypot(table.c_re, table.c_im),
                ghi_lo=ghi_lo, ghi_hi=ghi_hi, glo_lo=glo_lo, glo_hi=glo_hi, psi_lo=psi_lo, psi_hi=psi_hi)


def table_from_fields(f: dict, seed: int = -1) -> ZeroTableData:
    """ZeroTableData from reference fields (G exact; c = alpha e^{-2 pi i psi/2^128} in FP64)."""
    G3 = G3_from_ghi_glo(f["ghi_lo"], f["ghi_hi"], f["glo_lo"], f["glo_hi"])
    if "alpha" in f:
        alpha = f["alpha"]
    else:
        raise FormatError("fields carry no |c| (alpha)")
    c_re, c_im = c_from_alpha_psi(alpha, f["psi_lo"], f["psi_hi"])
    gamma = np.ascontiguousarray(f["gamma"], np.float64)
    if gamma.shape[0] > 1 and not np.all(np.diff(gamma) > 0):
        raise FormatError("gamma is not strictly increasing")
    return ZeroTableData(G3=G3, gamma=gamma, c_re=np.ascontiguousarray(c_re), c_im=np.ascontiguousarray(c_im),
                         seed=seed)


# ------------------------------------------------------------------ zeros_600k.bin

def read_zeros_600k(path: str) -> dict:
    size = os.path.getsize(path)
    with open(path, "rb") as fh:
        head = fh.read(8)
        if len(head) != 8:
            raise FormatError(f"{path}: no header")
        n = struct.unpack("<Q", head)[0]
        if size != 8 + n * (16 + 48):
            raise FormatError(f"{path}: size {size} does not match n={n}")
        gamma = np.frombuffer(fh.read(n * 8), dtype=np.float64).copy()
        alpha = np.frombuffer(fh.read(n * 8), dtype=np.float64).copy()
        raw = np.frombuffer(fh.read(n * 48), dtype=u).reshape(n, 6)
    out = {k: np.ascontiguousarray(raw[:, i]) for i, k in enumerate(_KEYS)}
    out.update(n=n, gamma=gamma, alpha=alpha)
    return out


def write_zeros_600k(path: str, f: dict) -> None:
    rec = np.stack([np.asarray(f[k], u) for k in _KEYS], axis=1)
    tmp = path + ".tmp"
    with open(tmp, "wb") as fh:
        fh.write(struct.pack("<Q", int(f["n"])))
        fh.write(np.ascontiguousarray(f["gamma"], np.float64).tobytes())
        fh.write(np.ascontiguousarray(f["alpha"], np.float64).tobytes())
        fh.write(np.ascontiguousarray(rec).tobytes())
    os.replace(tmp, path)


# ------------------------------------------------------------------ zeros.bin

ZEROS_BIN_K = 3e-9     # the Gaussian folded into two_astar (search/path1_build_zeros_100k.py:59)


def read_zeros_bin(path: str) -> dict:
    size = os.path.getsize(path)
    with open(path, "rb") as fh:
        head = fh.read(4)
        if len(head) != 4:
            raise FormatError(f"{path}: no header")
        n = struct.unpack("<i", head)[0]
        if n < 0 or size != 4 + n * 64:
            raise FormatError(f"{path}: size {size} does not match n={n}")
        two_astar = np.frombuffer(fh.read(n * 8), dtype=np.float64).copy()
        gamma = np.frombuffer(fh.read(n * 8), dtype=np.float64).copy()
        out = {k: np.frombuffer(fh.read(n * 8), dtype=u).copy() for k in _KEYS}
    out.update(n=n, gamma=gamma, two_astar=two_astar)
    # alpha = |c| from the folded weight (exact up to FP64 rounding while the weight is normal)
    out["alpha"] = two_astar / (2.0 * np.exp(-ZEROS_BIN_K * gamma * gamma))
    return out


def write_zeros_bin(path: str, f: dict) -> None:
    two_astar = np.asarray(f.get("two_astar", 2.0 * np.asarray(f["alpha"]) * np.exp(-ZEROS_BIN_K * np.asarray(f["gamma"]) ** 2)))
    tmp = path + ".tmp"
    with open(tmp, "wb") as fh:
        fh.write(struct.pack("<i", int(f["n"])))
        fh.write(np.ascontiguousarray(two_astar, np.float64).tobytes())
        fh.write(np.ascontiguousarray(f["gamma"], np.float64).tobytes())
        for k in _KEYS:
            fh.write(np.ascontiguousarray(f[k], u).tobytes())
    os.replace(tmp, path)


# ------------------------------------------------------------------ zero cache text (Arb balls)

_BALL = re.compile(r"^\s*\[\s*([+\-]?[0-9.]+(?:[eE][+\-]?\d+)?)\s*\+/-\s*([0-9.]+(?:[eE][+\-]?\d+)?)\s*\]\s*$")


def parse_ball(s: str):
    """(mid decimal string, radius float) of an Arb ball string '[mid +/- rad]' or a plain number."""
    m = _BALL.match(s)
    if m:
        return m.group(1), float(m.group(2))
    float(s)            # raises on garbage
    return s.strip(), 0.0


@dataclass
class ZeroCacheRadii:
    """Radii of the certified balls: gamma, Re c, Im c (per zero, FP64 upper bounds)."""
    gamma: np.ndarray
    c_re: np.ndarray
    c_im: np.ndarray


def read_zero_cache(paths) -> tuple[ZeroTableData, ZeroCacheRadii]:
    """Zero-cache text files (in order) -> table + radii.  G = gamma_mid / 2pi as 64.128
    fixed point (floor), c = ball midpoints rounded to FP64; the radii include those roundings."""
    import mpmath as mp

    if isinstance(paths, str):
        paths = [paths]
    gs, crs, cis, rg, rr, ri = [], [], [], [], [], []
    for p in paths:
        for ln, line in enumerate(open(p), 1):
            parts = line.rstrip("\n").split("\t")
            if len(parts) != 4:
                raise FormatError(f"{p}:{ln}: expected 4 tab-separated fields")
            (g, gr), (a, ar), (b, br) = (parse_ball(x) for x in parts[:3])
            gs.append(g); crs.append(a); cis.append(b)
            rg.append(gr); rr.append(ar); ri.append(br)
    n = len(gs)
    G3 = np.zeros((n, 3), u)
    gamma = np.zeros(n); c_re = np.zeros(n); c_im = np.zeros(n)
    rad_g = np.array(rg); rad_r = np.array(rr); rad_i = np.array(ri)
    with mp.workprec(400):
        two_pi = 2 * mp.pi
        for j in range(n):
            gm = mp.mpf(gs[j])
            Gf = int(mp.floor(gm / two_pi * mp.mpf(2) ** 128))
            if Gf >> 160:
                raise FormatError(f"zero {j}: gamma too large")
            G3[j] = (Gf >> 128, (Gf >> 64) & ((1 << 64) - 1), Gf & ((1 << 64) - 1))
            gamma[j] = float(gm)
            c_re[j], c_im[j] = float(mp.mpf(crs[j])), float(mp.mpf(cis[j]))
            # add the roundings of the stored values to the radii: G is floored to 2^-128
            # (2pi 2^-128 in gamma), c is rounded to FP64
            rad_g[j] += 2 * math.pi * 2.0 ** -128
            rad_r[j] += float(abs(mp.mpf(c_re[j]) - mp.mpf(crs[j])))
            rad_i[j] += float(abs(mp.mpf(c_im[j]) - mp.mpf(cis[j])))
    if n > 1 and not np.all(np.diff(gamma) > 0):
        raise FormatError("zero cache not strictly increasing")
    t = ZeroTableData(G3=G3, gamma=gamma, c_re=c_re, c_im=c_im, seed=-1)
    return t, ZeroCacheRadii(rad_g * (1 + 2 ** -50), rad_r * (1 + 2 ** -50), rad_i * (1 + 2 ** -50))


def term_radius(radii: ZeroCacheRadii, table: ZeroTableData, v: float) -> np.ndarray:
    """Per-zero bound on |c e^{i gamma v} - c_stored e^{i gamma_stored v}| implied by the ball
    radii (|dc| + |c| |v| dgamma), for the certified evaluation's term_rad."""
    dc = np.hypot(radii.c_re, radii.c_im)
    cabs = np.hypot(table.c_re, table.c_im) + dc
    return (dc + cabs * abs(v) * radii.gamma) * (1 + 2 ** -48)


def write_zero_cache(path: str, table: ZeroTableData, dps: int = 45) -> None:
    """Zero-cache text lines for a table whose G and c are exact (synthetic): gamma = 2pi G to
    dps digits with a radius covering the decimal rounding, c written exactly."""
    import mpmath as mp

    lines = []
    with mp.workprec(int(dps * 3.33) + 64):
        two_pi = 2 * mp.pi
        for j in range(table.n):
            gi, g1, g2 = (int(x) for x in table.G3[j])
            G = mp.mpf((gi << 128) | (g1 << 64) | g2) / mp.mpf(2) ** 128
            g = two_pi * G
            gstr = mp.nstr(g, dps + 5, strip_zeros=False)
            rad = abs(mp.mpf(gstr) - g) * 2 + mp.mpf(10) ** (-(dps + 3))
            lines.append(f"[{gstr} +/- {mp.nstr(rad, 3)}]\t[{float(table.c_re[j])!r} +/- 0]\t"
                         f"[{float(table.c_im[j])!r} +/- 0]\t0.0\n")
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        fh.writelines(lines)
    os.replace(tmp, path)
