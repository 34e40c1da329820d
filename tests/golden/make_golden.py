"""Generates the golden fixtures in this directory (run once; the outputs are committed).

    python tests/golden/make_golden.py [--skip-full-ball]

small_plain.json    64 candidates x 10,000 synthetic zeros (table seed 1, candidate seed 2),
                    k = 3e-9, T = inf:
                      * the reference's own compiled evaluator (oracle/_ref/libpath1_eval.so from
                        search/path1_eval_fast.cpp): compute_peak_AB + h0 = sum w A
                        (polish_peaks_with_weights with grid_steps = 0) and its polished h/ddy with
                        the drivers' settings (grid_half_width 2.5e-4, 40 steps);
                      * the binary128 oracle's K2, dK2/ddelta, dK2/dk (hi + lo doubles);
                      * mpmath interval balls of K2 and of dK2/ddelta, dK2/dk for 4 candidates
                        (220 bits);
                      * exact phases floor(frac(v G) 2^128) for 16 (candidate, zero) pairs.
zerodata_ref.json   the reference enumerator's own ZeroData (search/fast_mertens_enum.cpp, compiled
                    by oracle/Makefile through oracle/zerodata_ref.cpp) on synth.enumerator_table()
                    (40,000 zeros, c scaled by 3): fast_screen decisions of 16,384 leaves and
                    polish (h, dy) of 48 hits (--only zerodata writes just this one).
peak2_full_ball.json the interval ball of K2 at the reference's Peak2 point over all 2,325,572
                    synthetic zeros below 1.3e6 (table seed 1), k = 1.5e-10, as exact rational
                    endpoints (mpmath iv at 220 bits, summed in 64 worker processes' chunks),
                    plus the binary128 value.
path1_polish.json   the reference's own polish_single_peak and fast_polish_batch_blas
                    (search/path1_kernel_opt.py:94-221, the two function bodies executed with
                    numpy; the module itself needs gmpy2 and its shared library to import) on
                    A/B of 64 candidates (seed 3) x the first 2,000 zeros of table seed 1 from the
                    binary128 oracle, with the JP weight and exp(-3e-9 gamma^2); and 16 exact
                    A/B pairs at 256 bits (mpmath), the compute_exact_mpfr_AB contract (:71-91).
Each fixture records the SHA-256 of the table arrays so a generator change is detected.
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

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from mertens_bound_b200 import synth  # noqa: E402


def table_sha(t) -> str:
    h = hashlib.sha256()
    for a in (t.G3, t.gamma, t.c_re, t.c_im):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def frac_str(q: Fraction) -> str:
    return f"{q.numerator}/{q.denominator}"


def small_fixture():
    from oracle.interval import bounds, k2_ball
    from oracle.oracle import Oracle, RefLib, phase128_bigint, reference_candidates, reference_format

    t = synth.make_table(10_000, seed=1)
    c = synth.make_candidates(64, seed=2)
    k = 3e-9
    O = Oracle()
    hi, lo = O.k2(c, t, k, t.n)
    out = {"table": {"n": t.n, "seed": 1, "sha256": table_sha(t)}, "candidates": {"seed": 2, "P": 64},
           "k": k, "T": "inf",
           "v_int": [str(int(x)) for x in c.v_int], "v_frac": [str(int(x)) for x in c.v_frac],
           "oracle_k2": {"val": [[float(hi[p, 0]), float(lo[p, 0])] for p in range(64)],
                         "dd": [[float(hi[p, 1]), float(lo[p, 1])] for p in range(64)],
                         "dk": [[float(hi[p, 2]), float(lo[p, 2])] for p in range(64)]}}
    if RefLib.available():
        R = RefLib()
        A, B = R.peak_AB(reference_candidates(c), reference_format(t))
        w = np.exp(-k * t.gamma ** 2)
        h0, _, _ = R.polish(A, B, t.gamma, w, 2.5e-4, 0)
        hu, hp, dp = R.polish(A, B, t.gamma, w, 2.5e-4, 40)
        out["reference_evaluator"] = {"h0": [float(x) for x in h0], "h_pol": [float(x) for x in hp],
                                      "ddy_pol": [float(x) for x in dp],
                                      "source": "search/path1_eval_fast.cpp compiled by oracle/Makefile"}
    balls, dballs = [], []
    for p in range(4):
        val, dd, dk = k2_ball(c.v_int[p], c.v_frac[p], 0.0, t.G3, t.c_re, t.c_im, k, t.n)
        a, b = bounds(val)
        balls.append([frac_str(a), frac_str(b)])
        dballs.append({"dd": [frac_str(x) for x in bounds(dd)], "dk": [frac_str(x) for x in bounds(dk)]})
    out["interval_balls_first4"] = balls
    out["derivative_balls_first4"] = dballs
    pairs = []
    rng = np.random.default_rng(7)
    for _ in range(16):
        p, j = int(rng.integers(64)), int(rng.integers(t.n))
        h, l = phase128_bigint(c.v_int[p], c.v_frac[p], t.G3[j])
        pairs.append({"p": p, "j": j, "hi": str(h), "lo": str(l)})
    out["exact_phases"] = pairs
    return out


# The reference checkout: --ref, or the environment variable MB_REFERENCE_DIR, else a directory
# named `reference` beside this repository.
REF_DIR = os.environ.get("MB_REFERENCE_DIR",
                         os.path.abspath(os.path.join(HERE, "..", "..", "..", "reference")))


def reference_path1_functions():
    """polish_single_peak and fast_polish_batch_blas from the reference source, executed in a
    namespace holding only numpy and math."""
    import ast
    tree = ast.parse(open(os.path.join(REF_DIR, "search", "path1_kernel_opt.py")).read())
    keep = [n for n in tree.body if isinstance(n, ast.FunctionDef)
            and n.name in ("polish_single_peak", "fast_polish_batch_blas")]
    ns = {"np": np, "math": math}
    exec(compile(ast.Module(body=keep, type_ignores=[]), "path1_kernel_opt.py", "exec"), ns)
    return ns["polish_single_peak"], ns["fast_polish_batch_blas"]


def path1_weights(gamma):
    u = gamma / gamma[-1]
    return {"jp": (1.0 - u) * np.cos(np.pi * u) + np.sin(np.pi * u) / np.pi,
            "g3e-9": np.exp(-3e-9 * gamma * gamma)}


def path1_fixture():
    import mpmath
    from oracle.oracle import Oracle

    t = synth.make_table(10_000, seed=1)
    c = synth.make_candidates(64, seed=3)
    n = 2000
    A, B = Oracle().exact_AB(c, t, n)
    single, batch = reference_path1_functions()
    g = t.gamma[:n]
    out = {"table": {"n": t.n, "seed": 1, "sha256": table_sha(t)}, "candidates": {"seed": 3, "P": 64},
           "n_zeros": n, "AB_sha256": hashlib.sha256(A.tobytes() + B.tobytes()).hexdigest(),
           "source": "search/path1_kernel_opt.py:94-221 executed on oracle A/B"}
    for name, w in path1_weights(g).items():
        rows = [single(A[p], B[p], g, w, n_zeros=n, grid_hw=4e-5, grid_steps=40) for p in range(8)]
        hu, hp, dp = batch(A, B, g, w)
        out[name] = {"single_first8": [[float(x) for x in r] for r in rows],
                     "batch": {"h_unpol": [float(x) for x in hu], "h_pol": [float(x) for x in hp],
                               "ddy_pol": [float(x) for x in dp]}}
    mpmath.mp.prec = 256
    pairs = []
    rng = np.random.default_rng(11)
    for _ in range(16):
        p, j = int(rng.integers(64)), int(rng.integers(n))
        v = mpmath.mpf(int(c.v_int[p])) + mpmath.mpf(int(c.v_frac[p])) / 2 ** 64
        G = mpmath.mpf(int(t.G3[j, 0])) + mpmath.mpf(int(t.G3[j, 1])) / 2 ** 64 + mpmath.mpf(int(t.G3[j, 2])) / 2 ** 128
        th = 2 * mpmath.pi * G * v
        cr, ci = mpmath.mpf(float(t.c_re[j])), mpmath.mpf(float(t.c_im[j]))
        co, si = mpmath.cos(th), mpmath.sin(th)
        pairs.append({"p": p, "j": j, "A": float(2 * (cr * co - ci * si)), "B": float(2 * (cr * si + ci * co))})
    out["exact_AB_pairs_256bit"] = pairs
    return out


_WORKER = {}


def _init_worker():
    sys.path.insert(0, ROOT)
    from mertens_bound_b200 import synth as S
    _WORKER["t"] = S.make_table(2_325_572, seed=1)
    _WORKER["c"] = S.peak2_candidate()


def _ball_chunk(args):
    from oracle.interval import bounds, k2_ball
    j0, j1 = args
    t, c = _WORKER["t"], _WORKER["c"]
    val, _, _ = k2_ball(c.v_int[0], c.v_frac[0], 0.0, t.G3[j0:j1], t.c_re[j0:j1], t.c_im[j0:j1], 1.5e-10, j1 - j0)
    a, b = bounds(val)
    return j0, frac_str(a), frac_str(b)


def full_ball_fixture(workers: int):
    import multiprocessing as mp
    from oracle.oracle import Oracle

    t = synth.make_table(2_325_572, seed=1)
    c = synth.peak2_candidate()
    n = t.n
    edges = np.linspace(0, n, 513).astype(int)
    tasks = [(int(a), int(b)) for a, b in zip(edges[:-1], edges[1:])]
    t0 = time.time()
    with mp.get_context("spawn").Pool(workers, initializer=_init_worker) as pool:
        parts = pool.map(_ball_chunk, tasks, chunksize=1)
    lo = sum((Fraction(a) for _, a, _ in parts), Fraction(0))
    hi = sum((Fraction(b) for _, _, b in parts), Fraction(0))
    qhi, qlo = Oracle().k2(c, t, 1.5e-10, n)
    return {"table": {"n": n, "seed": 1, "sha256": table_sha(t)}, "v": synth.PEAK2_STR,
            "v_int": str(int(c.v_int[0])), "v_frac": str(int(c.v_frac[0])), "k": 1.5e-10, "T0": 1.3e6,
            "ball_lo": frac_str(lo), "ball_hi": frac_str(hi), "ball_width": float(hi - lo),
            "oracle_k2": [float(qhi[0, 0]), float(qlo[0, 0])],
            "method": "mpmath iv at 220 bits per term over 512 zero ranges, exact rational sum",
            "seconds": round(time.time() - t0, 1)}


def zerodata_fixture():
    """The reference enumerator's own ZeroData (search/fast_mertens_enum.cpp:27-277, compiled from
    its source into oracle/_ref/libzerodata_ref.so) on synth.enumerator_table() written as a
    zeros.bin: fast_screen decisions of 16,384 random leaves and polish (h, dy) of 48 hits (the 32
    leaves of largest |h| among the first 4,096, which run all five stages, and 16 others)."""
    import tempfile
    from mertens_bound_b200 import formats
    from oracle.oracle import MASK64, ZeroDataRef

    t = synth.enumerator_table()
    f = formats.reference_fields(t, exact_psi=True)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "zeros.bin")
        formats.write_zeros_bin(path, f)
        Z = ZeroDataRef(path)
        x = synth.leaves_x(16384, seed=21)
        x_lo = np.array([v & MASK64 for v in x], np.uint64)
        x_hi = np.array([v >> 64 for v in x], np.uint64)
        passed = Z.fast_screen(x_lo, x_hi)
        h, dy = Z.polish(x_lo[:4096], x_hi[:4096])
        deep = np.argsort(-np.abs(h), kind="stable")[:32]
        rest = np.setdiff1d(np.arange(4096), deep)
        other = np.random.default_rng(22).choice(rest, 16, replace=False)
        sel = np.concatenate([np.sort(deep), np.sort(other)])
        Z.close()
    xs = np.array([[v & MASK64, v >> 64] for v in x], np.uint64)
    return {"table": {"n": t.n, "seed": 1, "c_scale": synth.ENUM_C_SCALE, "sha256": table_sha(t)},
            "zeros_bin": "formats.reference_fields(exact_psi=True) -> formats.write_zeros_bin "
                         "(two_astar = 2|c| exp(-3e-9 gamma^2))",
            "leaves": {"count": 16384, "seed": 21, "form": "x = floor(v 2^30) of synth.make_candidates",
                       "sha256": hashlib.sha256(xs.tobytes()).hexdigest()},
            "screen_pass_packbits_hex": np.packbits(passed).tobytes().hex(), "screen_passed": int(passed.sum()),
            "polish": [{"leaf": int(i), "x": str(x[i]), "h": float(h[i]), "dy": float(dy[i])} for i in sel],
            "source": "search/fast_mertens_enum.cpp ZeroData::load/fast_screen/polish via oracle/zerodata_ref.cpp"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--skip-full-ball", action="store_true")
    ap.add_argument("--workers", type=int, default=os.cpu_count())
    ap.add_argument("--only", choices=["zerodata"], default=None,
                    help="write only this fixture (zerodata: zerodata_ref.json, needs oracle/_ref built from "
                         "the reference source)")
    ap.add_argument("--ref", default=None, help="the reference checkout (default: MB_REFERENCE_DIR or "
                                                "../reference beside the repository)")
    a = ap.parse_args()
    global REF_DIR
    if a.ref:
        REF_DIR = os.path.abspath(a.ref)
    if a.only == "zerodata":
        with open(os.path.join(HERE, "zerodata_ref.json"), "w") as f:
            json.dump(zerodata_fixture(), f, indent=1)
        print("wrote zerodata_ref.json", flush=True)
        return
    with open(os.path.join(HERE, "small_plain.json"), "w") as f:
        json.dump(small_fixture(), f, indent=1)
    print("wrote small_plain.json", flush=True)
    with open(os.path.join(HERE, "path1_polish.json"), "w") as f:
        json.dump(path1_fixture(), f, indent=1)
    print("wrote path1_polish.json", flush=True)
    if not a.skip_full_ball:
        with open(os.path.join(HERE, "peak2_full_ball.json"), "w") as f:
            json.dump(full_ball_fixture(a.workers), f, indent=1)
        print("wrote peak2_full_ball.json", flush=True)


if __name__ == "__main__":
    main()
