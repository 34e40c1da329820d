"""Multi-GPU evaluation: one process per GPU with torch.distributed (NCCL over NVLink/NVSwitch).

Two ways the K2 sum splits, both exact partitions of the work:
  * candidate sharding -- candidates are independent; each rank evaluates a contiguous slice
    over the whole table and no collective is needed on the data path (bench.py's weak scaling);
    `gather_candidates` collects the slices when the caller wants them on every rank.
  * zero-range sharding -- for few candidates (the certified P = 1 case, small groups): each rank
    sums a contiguous zero range [j0, j1) of every group (mb_plan_set_zero_range /
    mb_k2_certified_range) and the partial sums are combined:
      - point values and gradients with one all_reduce(SUM) of the (val, dd, dk) partials;
      - certified intervals by all-gathering each rank's [lo, hi] and adding the endpoints in
        exact rational arithmetic, so the combined interval is still a rigorous enclosure
        (a floating-point all_reduce would round the lower end up).
The reference has no collectives; its batches go through a process pool and are reduced
serially (certification/certify_K2.py:160-192).
"""
from __future__ import annotations

from fractions import Fraction
from typing import Callable

import numpy as np


def shard_range(n: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous, balanced [start, end) of n items for `rank` of `world` (an exact partition)."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError("bad shard request")
    q, r = divmod(n, world)
    start = rank * q + min(rank, r)
    return start, start + q + (1 if rank < r else 0)


def _dist():
    import torch.distributed as dist
    return dist


def allreduce_sum(x: np.ndarray, device=None) -> np.ndarray:
    """Sum of x over all ranks (float64), through torch.distributed (NCCL on GPU, gloo on CPU)."""
    import torch
    dist = _dist()
    t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64).copy())
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def gather_candidates(local: np.ndarray, device=None) -> np.ndarray:
    """Concatenate every rank's slice (rank order) on every rank."""
    import torch
    dist = _dist()
    world = dist.get_world_size()
    t = torch.from_numpy(np.ascontiguousarray(local, dtype=np.float64).copy())
    if device is not None:
        t = t.to(device)
    n = torch.tensor([t.shape[0]], dtype=torch.int64, device=t.device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n)
    m = int(max(s.item() for s in sizes))
    pad = torch.zeros((m,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
    pad[: t.shape[0]] = t
    parts = [torch.zeros_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad)
    return np.concatenate([p[: int(s.item())].cpu().numpy() for p, s in zip(parts, sizes)])


def combine_intervals(local_lo: np.ndarray, local_hi: np.ndarray) -> list[tuple[Fraction, Fraction]]:
    """Exact sum over ranks of per-candidate intervals [lo, hi] (rigorous enclosure)."""
    dist = _dist()
    world = dist.get_world_size()
    mine = [(float(a), float(b)) for a, b in zip(local_lo, local_hi)]
    allp = [None] * world
    dist.all_gather_object(allp, mine)
    out = []
    for p in range(len(mine)):
        lo = sum((Fraction(r[p][0]) for r in allp), Fraction(0))
        hi = sum((Fraction(r[p][1]) for r in allp), Fraction(0))
        out.append((lo, hi))
    return out


def zero_sharded_value(eval_range: Callable[[int, int], np.ndarray], n_use: int, device=None) -> np.ndarray:
    """(P, 3) totals of (val, dd, dk) where eval_range(j0, j1) returns this rank's partials."""
    dist = _dist()
    j0, j1 = shard_range(n_use, dist.get_world_size(), dist.get_rank())
    return allreduce_sum(eval_range(j0, j1), device)


def zero_sharded_certified(eval_range: Callable[[int, int], tuple[np.ndarray, np.ndarray]], n_use: int):
    """Rigorous per-candidate enclosures where eval_range(j0, j1) returns (lo, hi) arrays."""
    dist = _dist()
    j0, j1 = shard_range(n_use, dist.get_world_size(), dist.get_rank())
    lo, hi = eval_range(j0, j1)
    return combine_intervals(lo, hi)


# ------------------------------------------------------------------ GPU evaluators

def gpu_value_evaluator(table, cands, k: float, T: float, tol: float = 1e-10):
    """eval_range for zero_sharded_value on this rank's GPU (chosen-form plan on a zero range)."""
    from . import k2
    plan = k2.Plan(table, [cands.n], [k], [T], tol=tol)

    def ev(j0: int, j1: int) -> np.ndarray:
        from ._lib import check, lib
        check(lib().mb_plan_set_zero_range(plan.handle, int(j0), int(j1)))
        val, dd, dk = plan.run(cands)
        return np.stack([val, dd, dk], axis=1)
    return ev


def gpu_certified_evaluator(table, cands, k_str: str, v_rad=None):
    """eval_range for zero_sharded_certified (interval kernel on a zero range)."""
    from . import certify
    from ._lib import check, lib, ptr
    klo, khi = certify.k_interval(k_str)
    vi = np.ascontiguousarray(cands.v_int, np.uint64)
    vf = np.ascontiguousarray(cands.v_frac, np.uint64)
    vr = None if v_rad is None else np.ascontiguousarray(np.broadcast_to(v_rad, vi.shape), np.float64)

    def ev(j0: int, j1: int):
        lo, hi = np.empty(vi.shape[0]), np.empty(vi.shape[0])
        check(lib().mb_k2_certified_range(table.handle, vi.shape[0], ptr(vi), ptr(vf), ptr(vr), klo, khi, int(j0),
                                          int(j1), None, ptr(lo), ptr(hi), None))
        return lo, hi
    return ev
