"""Certified K2 with the contract of certification/certify_K2.py, on the GPU interval kernel.

    python -m mertens_bound_b200.certify [--v V] [--k K] [--T0 T0] [--table FILE] [--out CERT.json]

certify_K2.py sums 2 e^{-k g^2} Re(c e^{i g v}) in Arb balls over 9,303 batches of 250 zeros in a
process pool (work(), :100-133) and reduces the batch balls serially (:176-207).  Here every
batch is one call of mb_k2_certified_range (directed-rounding interval arithmetic, the table's
exact G and c, v and k given as decimal strings and enclosed: v by its 64.64 floor plus a radius,
k by its two neighbouring doubles).  The reduction, contiguity/order checks, key-bound batch
cache and certificate fields follow the reference so check_theorem.py can read the result; the
certificate's schema is "b200-1" (the reference's schema 2 also binds FLINT versions, which do
not apply here).  Failures raise CertificationError (nonzero exit from the CLI), also under -O.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import math
import os
import sys
import time
from fractions import Fraction

import numpy as np

from . import k2, synth
from ._lib import K2Error, check, lib, ptr

SCHEMA = "b200-1"
K_STR = "1.5e-10"
V_STR = synth.PEAK2_STR
T0_STR = "1300000"
N_HI = 600000
BATCH = 250
HERE = os.path.dirname(os.path.abspath(__file__))
CODE = [os.path.join(HERE, "certify.py"), os.path.join(HERE, "csrc", "k2_certified.cu"),
        os.path.join(HERE, "csrc", "k2_common.cuh"), os.path.join(HERE, "csrc", "poly_coeffs.h")]


class CertificationError(RuntimeError):
    pass


def require(cond, msg):
    if not cond:
        raise CertificationError(msg)


# ------------------------------------------------------------------ exact enclosures and balls

def k_interval(k_str: str) -> tuple[float, float]:
    """The doubles k_lo <= k <= k_hi around a decimal k (equal when k is a double)."""
    q = Fraction(k_str)
    require(q >= 0, f"k={k_str} must be >= 0")
    d = float(q)
    lo = d if Fraction(d) <= q else math.nextafter(d, -math.inf)
    hi = d if Fraction(d) >= q else math.nextafter(d, math.inf)
    return lo, hi


def v_point(v_str: str) -> tuple[int, int, float]:
    """(v_int, v_frac, v_rad): v = v_int + v_frac 2^-64 + e with 0 <= e <= v_rad."""
    q = Fraction(v_str)
    require(0 <= q < 2 ** 64, f"v={v_str} out of range")
    vi = int(q)
    vf = int((q - vi) * (1 << 64))
    rem = q - vi - Fraction(vf, 1 << 64)
    rad = float(rem)
    if Fraction(rad) < rem:
        rad = math.nextafter(rad, math.inf)
    return vi, vf, rad


def ball(lo, hi, digits: int = 20) -> str:
    """Ball string '[mid +/- rad]' whose interval contains [lo, hi] (exact rationals)."""
    lo, hi = Fraction(lo), Fraction(hi)
    require(lo <= hi, "empty interval")
    mid = (lo + hi) / 2
    if mid == 0:
        exp10 = 0
    else:
        exp10 = math.floor(math.log10(abs(float(mid)))) if float(mid) != 0 else -300
    scale = Fraction(10) ** (digits - 1 - exp10)
    m = Fraction(round(mid * scale)) / scale
    r = max(hi - m, m - lo)
    rf = float(r)
    if Fraction(rf) < r:
        rf = math.nextafter(rf, math.inf)
    rs = f"{rf:.3e}"
    while Fraction(rs) < r:                   # the printed radius must still cover
        rf = math.nextafter(float(rs), math.inf) * (1 + 1e-3)
        rs = f"{rf:.3e}"
    ms = _decimal(m, digits + 3)
    return f"[{ms} +/- {rs}]"


def _decimal(q: Fraction, sig: int) -> str:
    if q == 0:
        return "0"
    neg = q < 0
    q = abs(q)
    e = math.floor(math.log10(float(q)))
    scale = Fraction(10) ** (sig - 1 - e)
    n = round(q * scale)
    s = str(n)
    point = len(s) - (sig - 1 - e)
    if point <= 0:
        s = "0." + "0" * (-point) + s
    elif point >= len(s):
        s = s + "0" * (point - len(s))
    else:
        s = s[:point] + "." + s[point:]
    return ("-" if neg else "") + s


def ball_bounds(s: str) -> tuple[Fraction, Fraction]:
    from .formats import parse_ball
    mid, rad = parse_ball(s)
    return Fraction(mid) - Fraction(rad), Fraction(mid) + Fraction(rad)


# ------------------------------------------------------------------ versions and cache keys

def file_hash(*paths) -> str:
    h = hashlib.sha256()
    for p in paths:
        with open(p, "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def table_hash(data) -> str:
    h = hashlib.sha256()
    for a in (data.G3, data.gamma, data.c_re, data.c_im):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def versions() -> dict:
    import platform
    import ctypes
    out = {"python": platform.python_version(), "libmertens_k2_abi": lib().mb_abi_version()}
    try:
        rt = ctypes.c_int()
        ctypes.CDLL("libcudart.so").cudaRuntimeGetVersion(ctypes.byref(rt))
        out["cuda_runtime"] = rt.value
    except OSError:
        pass
    return out


def cache_tag(params: dict, table_sha: str) -> str:
    blob = json.dumps({"params": params, "schema": SCHEMA, "versions": versions(), "table": table_sha,
                       "code": file_hash(*CODE)}, sort_keys=True)
    return hashlib.sha256(blob.encode()).hexdigest()[:16]


# ------------------------------------------------------------------ batch work (certify_K2.work)

def certified_range(table: k2.ZeroTable, v_str: str, k_str: str, j0: int, j1: int, term_rad=None):
    """Enclosure [lo, hi] of the sum over zeros [j0, j1) and an upper bound of sum 2 w |c|."""
    vi, vf, vr = v_point(v_str)
    klo, khi = k_interval(k_str)
    a_vi, a_vf, a_vr = (np.array([vi], np.uint64), np.array([vf], np.uint64), np.array([vr]))
    lo, hi, ab = np.empty(1), np.empty(1), np.empty(1)
    tr = None if term_rad is None else np.ascontiguousarray(term_rad, np.float64)
    require(tr is None or tr.shape == (j1 - j0,), "term_rad must have one entry per zero of the range")
    check(lib().mb_k2_certified_range(table.handle, 1, ptr(a_vi), ptr(a_vf), ptr(a_vr), klo, khi, int(j0), int(j1),
                                      ptr(tr), ptr(lo), ptr(hi), ptr(ab)))
    require(np.isfinite(lo[0]) and np.isfinite(hi[0]) and lo[0] <= hi[0], f"non-finite partial sum at zero {j0 + 1}")
    return float(lo[0]), float(hi[0]), float(ab[0])


_TWO_PI_LO = Fraction("6.283185307179586476925286766559005768")    # 2pi rounded down to 36 digits
_TWO_PI_HI = _TWO_PI_LO + Fraction(1, 10 ** 36)


def gamma_ball(data, j: int) -> str:
    """Ball of gamma_j = 2pi G_j from the exact fixed-point G_j."""
    gi, g1, g2 = (int(x) for x in data.G3[j])
    G = Fraction((gi << 128) | (g1 << 64) | g2, 1 << 128)
    return ball(_TWO_PI_LO * G, _TWO_PI_HI * G, 30)


def work(table: k2.ZeroTable, data, args, term_rad=None) -> dict:
    """certify_K2.work: args = (n0, num, dps, k_str, v_str, outdir, tag, cache_only).  Zeros
    n0 .. n0+num-1 (1-based) of the table; the result is cached in outdir under a key-checked
    JSON file, like the reference (:102-107, :129-132)."""
    n0, num, dps, k_str, v_str, outdir, tag, cache_only = args
    path = os.path.join(outdir, f"{n0:08d}_{num}_{dps}.json")
    if not cache_only and os.path.exists(path):
        with open(path) as f:
            res = json.load(f)
        require(res.get("tag") == tag and res.get("n0") == n0 and res.get("num") == num and res.get("dps") == dps
                and res.get("k") == k_str and res.get("v") == v_str, f"cache payload {path} does not match its key")
        return res
    require(1 <= n0 and n0 - 1 + num <= table.n, f"batch {n0}..{n0 + num - 1} outside the table")
    if cache_only:
        return {"n0": n0, "num": num}
    lo, hi, ab = certified_range(table, v_str, k_str, n0 - 1, n0 - 1 + num, term_rad)
    res = {"tag": tag, "k": k_str, "v": v_str, "n0": n0, "num": num, "dps": dps,
           "S": ball(lo, hi, 25), "absS": ball(0, ab, 12),
           "g_first": gamma_ball(data, n0 - 1), "g_last": gamma_ball(data, n0 - 2 + num),
           "min_abs_zeta_prime": None,
           "max_term_rad": float(np.max(term_rad)) if term_rad is not None and len(term_rad) else 0.0}
    os.makedirs(outdir, exist_ok=True)
    tmp = path + f".tmp{os.getpid()}"
    with open(tmp, "w") as f:
        json.dump(res, f)
    os.replace(tmp, path)
    return res


def reduce_batches(results: list[dict], N: int, n_hi: int):
    """Contiguity and ordering checks and the interval sums (certify_K2.py:176-192)."""
    results = sorted(results, key=lambda r: r["n0"])
    require(results and results[0]["n0"] == 1 and sum(r["num"] for r in results) == N, "batches do not cover 1..N(T0)")
    for r1, r2 in zip(results, results[1:]):
        require(r1["n0"] + r1["num"] == r2["n0"], f"gap between batches at n={r2['n0']}")
        require(ball_bounds(r1["g_last"])[1] < ball_bounds(r2["g_first"])[0], f"batches not ordered by height at n={r2['n0']}")
    main = [Fraction(0), Fraction(0)]
    tail = [Fraction(0), Fraction(0)]
    tail_abs = Fraction(0)
    for r in results:
        lo, hi = ball_bounds(r["S"])
        dst = main if r["n0"] + r["num"] - 1 <= n_hi else tail
        dst[0] += lo
        dst[1] += hi
        if dst is tail:
            tail_abs += ball_bounds(r["absS"])[1]
    return main, tail, tail_abs


# ------------------------------------------------------------------ full certificate

def certify(data, v_str: str = V_STR, k_str: str = K_STR, T0_str: str = T0_STR, n_hi: int = N_HI,
            batch: int | None = None, outdir: str | None = None, term_rad=None, device: int = 0) -> dict:
    """Certificate dict for K2(v, T0, k) over all table zeros below T0."""
    t0 = time.time()
    T0 = float(Fraction(T0_str))
    params = {"k": k_str, "v": v_str, "T0": T0_str, "N_HI": n_hi, "BATCH": batch}
    tsha = table_hash(data)
    with k2.ZeroTable.from_data(data, device=device) as table:
        N = table.count_below(T0)
        require(N >= 1, "no zeros below T0")
        require(Fraction(float(data.gamma[N - 1])) < Fraction(T0_str), "table order")
        if N < data.n:
            g_n, g_n1 = Fraction(float(data.gamma[N - 1])), Fraction(float(data.gamma[N]))
            T0q = Fraction(T0_str)
            slack = Fraction(2) ** -40 * T0q                 # gamma_f64 is within 4 ulp of 2pi G
            delta = min(T0q - g_n, g_n1 - T0q) - slack
            require(delta > 0, "cutoff gap not certified positive")
            delta_ball = ball(delta, delta, 15)
        else:
            delta_ball = None                                 # the table ends below T0
        if batch:
            tag = cache_tag(params, tsha)
            outdir = outdir or os.path.join(os.getcwd(), "k2_chunks", tag)
            results = []
            for n0 in range(1, N + 1, batch):
                num = min(batch, N + 1 - n0)
                if n0 <= n_hi < n0 + num - 1:
                    raise CertificationError("BATCH must divide N_HI")
                tr = None if term_rad is None else term_rad[n0 - 1:n0 - 1 + num]
                results.append(work(table, data, (n0, num, 45 if n0 <= n_hi else 20, k_str, v_str, outdir, tag, False), tr))
            main, tail, tail_abs = reduce_batches(results, N, n_hi)
            manifest = hashlib.sha256("".join(json.dumps(r, sort_keys=True) for r in
                                              sorted(results, key=lambda r: r["n0"])).encode()).hexdigest()
        else:
            m = min(n_hi, N)
            lo, hi, _ = certified_range(table, v_str, k_str, 0, m, None if term_rad is None else term_rad[:m])
            main = [Fraction(lo), Fraction(hi)]
            if N > m:
                lo, hi, ab = certified_range(table, v_str, k_str, m, N, None if term_rad is None else term_rad[m:N])
                tail, tail_abs = [Fraction(lo), Fraction(hi)], Fraction(ab)
            else:
                tail, tail_abs = [Fraction(0), Fraction(0)], Fraction(0)
            manifest = None
    K2 = (main[0] + tail[0], main[1] + tail[1])
    cert = {
        "schema": SCHEMA, "params": params, "versions": versions(),
        "code_sha256": {os.path.basename(p): file_hash(p) for p in CODE}, "table_sha256": tsha,
        "k": k_str, "v": v_str, "T0": T0_str, "N_T0": int(N), "delta_lower": delta_ball,
        f"K2_main_(n<={n_hi})": ball(*main, 30), "K2_tail_ball": ball(*tail, 15),
        "K2_tail_abs_bound": ball(0, tail_abs, 12), "K2": ball(*K2, 30), "K2_lower_ball": ball(K2[0], K2[0], 25),
        "chunk_manifest_sha256": manifest,
        "method": "libmertens_k2 directed-rounding interval kernel (exact 64.128 phases, Taylor enclosures)",
        "N_T0_source": "count of table zeros below T0 (the reference certifies it with arb.zeta_nzeros)",
        "elapsed_s_this_run": round(time.time() - t0, 3),
    }
    return cert


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="Certified K2 on the GPU (certify_K2.py contract)")
    # certify_K2.py's command line: [workers] --v --k --out --cache-only (:137-142)
    ap.add_argument("workers", nargs="?", type=int, default=None,
                    help="accepted for certify_K2.py's command line; the GPU kernel needs no worker pool")
    ap.add_argument("--v", default=V_STR)
    ap.add_argument("--k", default=K_STR)
    ap.add_argument("--T0", default=T0_STR)
    ap.add_argument("--table", default=None, help="zero-cache .txt (default: synthetic zeros below T0)")
    ap.add_argument("--cache-dir", default=None,
                    help="directory of zero-cache files ({n0:08d}_{num}_{dps}.txt, read in name order)")
    ap.add_argument("--cache-only", action="store_true",
                    help="certify_K2.py's zero generation step: not part of this evaluator")
    ap.add_argument("--batch", type=int, default=0, help="certify in batches with a key-checked cache")
    ap.add_argument("--out", default="k2_certificate.json")
    a = ap.parse_args(argv)
    if a.cache_only:
        print("FAIL: --cache-only generates zeros (acb.zeta_zeros); this evaluator only reads zero caches",
              file=sys.stderr)
        return 2
    try:
        term_rad = None
        files = None
        if a.cache_dir:
            import glob
            files = sorted(glob.glob(os.path.join(a.cache_dir, "*.txt")))
            require(files, f"no zero-cache files in {a.cache_dir}")
        elif a.table:
            files = [a.table]
        if files:
            from . import formats
            data, radii = formats.read_zero_cache(files)
            term_rad = formats.term_radius(radii, data, float(Fraction(a.v)))
        else:
            # synthetic zeros a little beyond T0, so the gap around T0 can be certified
            data = synth.make_table_below(float(Fraction(a.T0)) * 1.01 + 100.0, seed=1)
        require(data.n >= 1 and data.count_below(float(Fraction(a.T0))) >= 1, "no zeros below T0")
        cert = certify(data, a.v, a.k, a.T0, batch=a.batch or None, term_rad=term_rad)
        print(json.dumps(cert, indent=2))
        with open(a.out, "w") as f:
            json.dump(cert, f, indent=2)
        return 0
    except (CertificationError, K2Error) as e:
        print(f"FAIL: {e}", file=sys.stderr)
        return 1


if __name__ == "__main__":
    sys.exit(main())
