"""Builds libmertens_k2.so in-tree from csrc/*.cu for sm_100a.

  python -m mertens_bound_b200.build [-v]

Objects go to mertens_bound_b200/_build/, the shared library to
mertens_bound_b200/libmertens_k2.so.  Only sources newer than their object are recompiled.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmertens_k2.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "-I", CSRC, "-I", INCLUDE]


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(INCLUDE, "mertens_k2.h"))
    return max(os.path.getmtime(h) for h in hs if os.path.exists(h))


def _compile(src: str, verbose: bool) -> tuple[str, str]:
    obj = os.path.join(BUILD, src[:-3] + ".o")
    cmd = [NVCC, *ARCH, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def ensure_poly_header():
    hdr = os.path.join(CSRC, "poly_coeffs.h")
    gen = os.path.join(CSRC, "gen_poly.py")
    if not os.path.exists(hdr) or os.path.getmtime(gen) > os.path.getmtime(hdr):
        out = subprocess.run([sys.executable, gen], capture_output=True, text=True, check=True).stdout
        with open(hdr, "w") as f:
            f.write(out)


def build_library(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    ensure_poly_header()
    hdr_t = _headers_mtime()
    todo = []
    for s in _sources():
        obj = os.path.join(BUILD, s[:-3] + ".o")
        src_t = max(os.path.getmtime(os.path.join(CSRC, s)), hdr_t)
        if force or verbose or not os.path.exists(obj) or os.path.getmtime(obj) < src_t:
            todo.append(s)
    logs = []
    if todo:
        with ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            for obj, log in ex.map(lambda s: _compile(s, verbose), todo):
                logs.append(log)
    objs = [os.path.join(BUILD, s[:-3] + ".o") for s in _sources()]
    if todo or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        tmp = LIB + ".tmp"
        cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    if verbose:
        print("\n".join(logs))
    return LIB


if __name__ == "__main__":
    print(build_library(verbose="-v" in sys.argv, force="-f" in sys.argv))
