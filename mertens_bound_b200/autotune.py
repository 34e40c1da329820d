"""Autotuner for the chosen-form plans.

The search space is the plan-wide tile configuration (mb_plan_configure) under each schedule
(mb_plan_set_schedule):
  light_cpt    candidates per thread in the light kernel: 2, 3, 4 (register budget 64/80/128,
               i.e. 4/3/2 CTAs per SM)
  nzw_shift    extra doublings of the warps that split one candidate set's zeros
  chunk_scale  work-item size relative to the automatic choice
  schedule     0: the two tier kernels concurrently, 1: one persistent kernel for both tiers,
               2: the same with all items ordered by estimated cost, 3: the same with one queue
               per tier (one CTA of each tier per SM)
Every configuration is timed on the device (median of `reps` runs, synthetic candidates) and the
fastest one is applied.  Results are cached per (GPU name, workload class) in a JSON file
($MB_AUTOTUNE_CACHE, default ~/.cache/mertens_k2/autotune.json); a workload class buckets the
candidate count, the zero counts and the heavy-tier fraction on a log scale.
"""
from __future__ import annotations

import json
import math
import os
import threading

from . import k2

SPACE = [(cpt, shift, scale) for cpt in (2, 3, 4) for shift in (0, 1) for scale in (0.5, 1.0, 2.0)]
SCHEDULES = (0, 1, 2, 3)
_lock = threading.Lock()


def cache_path() -> str:
    return os.environ.get("MB_AUTOTUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "mertens_k2",
                                                            "autotune.json"))


def device_name(device: int) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return f"cuda{device}"


def workload_key(plan: k2.Plan) -> str:
    heavy, light = plan.tier_terms()
    terms = max(heavy + light, 1.0)
    n_T = [plan.group_info(g)["n_T"] for g in range(len(plan.counts))]
    parts = [
        device_name(plan.table.device),
        f"G{len(plan.counts)}",
        f"P{round(math.log2(max(plan.P, 1)))}",
        f"N{round(math.log2(max(max(n_T), 1)))}",
        f"H{round(10 * heavy / terms)}",
    ]
    return "|".join(parts)


def _load() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(d: dict) -> None:
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + f".tmp{os.getpid()}"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass                                    # a read-only home just disables the cache


def _apply(plan: k2.Plan, cfg) -> None:
    plan.set_schedule(cfg[3] if len(cfg) > 3 else 0)
    plan.configure(*cfg[:3])


def autotune(plan: k2.Plan, reps: int = 3, use_cache: bool = True, space=SPACE, schedules=SCHEDULES) -> dict:
    """Pick and apply the fastest configuration (light_cpt, nzw_shift, chunk_scale, schedule);
    returns {config, ms, timings, cached}."""
    key = workload_key(plan)
    if use_cache:
        with _lock:
            hit = _load().get(key)
        if hit and len(hit["config"]) == 4:
            _apply(plan, hit["config"])
            return {"config": tuple(hit["config"]), "ms": hit["ms"], "timings": hit.get("timings", {}),
                    "cached": True, "key": key}
    timings = {}
    best = None
    for sched in schedules:
        plan.set_schedule(sched)
        if space == SPACE:                      # the library's own search over the same space
            import ctypes as C
            from ._lib import check, lib
            cpt, shift, scale, ms = C.c_int(), C.c_int(), C.c_double(), C.c_double()
            t = (C.c_double * len(SPACE))()
            check(lib().mb_plan_autotune(plan.handle, int(reps), C.byref(cpt), C.byref(shift), C.byref(scale),
                                         C.byref(ms), t))
            timings.update({f"{c}/{sh}/{sc}/{sched}": t[i] for i, (c, sh, sc) in enumerate(SPACE)})
            cand = ((cpt.value, shift.value, scale.value, sched), ms.value)
            if best is None or cand[1] < best[1]:
                best = cand
        else:
            for cfg in space:
                plan.configure(*cfg)
                ms = plan.time(reps)
                timings[f"{cfg[0]}/{cfg[1]}/{cfg[2]}/{sched}"] = ms
                if best is None or ms < best[1]:
                    best = ((*cfg, sched), ms)
    _apply(plan, best[0])
    if use_cache:
        with _lock:
            d = _load()
            d[key] = {"config": list(best[0]), "ms": best[1], "timings": timings}
            _store(d)
    return {"config": best[0], "ms": best[1], "timings": timings, "cached": False, "key": key}
