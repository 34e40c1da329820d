#!/usr/bin/env python3
"""Benchmark of the B200 K2 evaluator (one JSON line on rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (search-scoring shape): a synthetic table of all zeros below T0 = 3e5 (466,659
zeros), 4,096 candidate points v ~ 3.5e18 per GPU, k = 3e-9.  One step = K2 value and both
derivatives (dK2/ddelta, dK2/dk) for every candidate over every zero below T0, i.e.
4,096 x 466,659 zero-terms, with |K2 error| bounded a priori by tol = 1e-10.

Arms
  ours       the chosen form (tiered, batched plan) timed on the device with CUDA events,
             inputs resident in HBM; beside it the plain FP64 kernel (the ratio's denominator),
             the end-to-end number through the host-pointer API (pinned H2D + graph + D2H),
             a roofline of the dominant kernel, and the reference CPU evaluator timed on a
             bounded sample (cpu_baseline).
  reference  the reference's own CPU evaluator (search/path1_eval_fast.cpp compiled into
             oracle/_ref) on the same workload and metric, a bounded candidate sample per step.

Multi-GPU (torchrun): every rank evaluates its own 4,096 candidates over the same table
(candidates shard with no data-path collective: weak scaling); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "K₂ zero-terms/s (value+grad, |err|≤1e-10 vs Arb): chosen form vs plain FP64, 1 B200"
UNIT = "zero-terms/s"
T0, K_GAUSS, P_PER_GPU, TOL = 3e5, 3e-9, 4096, 1e-10
WORKLOAD = ("search_scoring: all 466,659 synthetic zeros below T0=3e5, 4,096 candidates v~3.5e18 "
            "per GPU, k=3e-9, K2 + dK2/ddelta + dK2/dk per candidate, a-priori |err| <= 1e-10")
# Per-launch DRAM bytes of the two tier kernels on this workload (light tier at each
# candidates-per-thread setting, its one-FMA fraction product), from one ncu capture of
# `bench.py --profile-case search` (dram__bytes_read.sum + dram__bytes_write.sum), and the
# executed thread instructions per zero-term of each kernel from the same capture
# (smsp__inst_executed.sum x 32 / zero-terms): the issue-slot side figure beside the pipe roofline.
LIGHT_DRAM_BYTES = {2: 16468736, 3: 16439040, 4: 16414976}
HEAVY_DRAM_BYTES = 2827264
TIERS_DRAM_BYTES = 19178240          # k2_tiers_kernel<4> (both tiers in one launch)
LIGHT_INST_PER_TERM = {2: 19.32, 3: 19.86, 4: 16.54}
HEAVY_INST_PER_TERM = 39.39
# Algorithmic operations per zero-term on each tier's binding pipe:
#   light tier, XU (MUFU) pipe: one sine and one cosine of the reduced phase;
#   heavy tier, FP64 pipe: 4 DFMA for the 2^-64-turn phase products, 1 add onto the rounding
#   constant, 1 FMA for the exact table remainder, 8 for the table sine/cosine (r^2, the sine
#   polynomial and product, the cosine product, two 2-FMA rotations) and 3 FMA accumulations of
#   K2, dK2/ddelta, dK2/dk.
LIGHT_MUFU_PER_TERM = 2
HEAVY_FP64_PER_TERM = 17
REF_SAMPLE_CANDS = 64
REF_TIMED_BUDGET_S = 200.0   # the reference arm's timed steps, at most (a bounded sample per step)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-workloads", action="store_true", help="skip the summary of the other workloads")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--profile-case", choices=["small", "search", "extras", "scoring"], default=None,
                    help="run a fixed case for ncu captures (no timing): 'small' = zeros below 1e5 x "
                         "2,048 candidates, all kernels of one plan run; 'search' = the bench workload, "
                         "each kernel launched alone once (plain; light tier at 2, 3, 4 candidates per "
                         "thread; heavy tier); 'extras' = certified, screen and polish kernels once each")
    return ap.parse_args()


# ---------------------------------------------------------------- clocks

CLOCK_QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


class ClockSampler:
    """SM clock and clock-event reasons of one GPU, read through NVML every `period` seconds on a
    background thread between construction and stop() (the timed region)."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, cuda_index: int, period: float = 0.002):
        import threading
        self.sm, self.masks, self.max_mhz, self.error = [], [], None, None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = self._handle(pynvml, cuda_index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
            self.bits = {name: getattr(pynvml, const) for name, const in self.REASONS}
        except Exception as e:                                   # no NVML: the line says so
            self.error = f"{type(e).__name__}: {e}"
            self.h = None
        self.t = threading.Thread(target=self._run, args=(period,), daemon=True)
        if self.h is not None:
            self._sample()                                       # at least one sample in the region
            self.t.start()

    @staticmethod
    def _handle(pynvml, cuda_index: int):
        """The NVML handle of CUDA device cuda_index (matched by PCI bus id, so a
        CUDA_VISIBLE_DEVICES mapping does not matter)."""
        try:
            import torch
            pr = torch.cuda.get_device_properties(cuda_index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(cuda_index)

    def _sample(self):
        nv = self.nv
        self.sm.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
        self.masks.append(int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)))

    def _run(self, period):
        while not self._stop.wait(period):
            try:
                self._sample()
            except Exception as e:
                self.error = f"{type(e).__name__}: {e}"
                return

    def stop(self) -> dict:
        if self.h is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "samples": 0, "reasons": [], "error": self.error}
        self._sample()
        self._stop.set()
        self.t.join(timeout=5)
        reasons = sorted(n for n, b in self.bits.items() if any(m & b for m in self.masks))
        out = {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": self.max_mhz, "samples": len(self.sm),
               "sm_mhz_min": min(self.sm), "reasons": reasons, "source": "NVML, sampled on a thread"}
        if self.error:
            out["error"] = self.error
        return out


# ---------------------------------------------------------------- reference CPU evaluator

def reference_rate(table, cands, k: float, n_use: int, seconds: float, steps: int | None = None,
                   per_step: int = REF_SAMPLE_CANDS):
    """Zero-terms/s of the reference's compute_peak_AB plus the value and gradient sums
    (h0 = sum w A as in path1_eval_fast.cpp:76-81, dK2/dv = -sum w gamma B,
    dK2/dk = -sum w gamma^2 A) as NumPy dots.  A step is per_step candidates in calls of
    REF_SAMPLE_CANDS candidates (the P x N A/B matrices of a whole step would not fit in memory);
    it runs `steps` steps, or steps until `seconds` have been spent."""
    from oracle.oracle import Oracle, RefLib, reference_candidates, reference_format

    reft = reference_format(table, n_use, exact_psi=False)
    w = np.exp(-k * table.gamma[:n_use] ** 2)
    wg, wg2 = w * table.gamma[:n_use], w * table.gamma[:n_use] ** 2
    if RefLib.available():
        R, kind, cores = RefLib(), "reference", 16           # team size fixed by the source (:33)
        peak_ab = lambda refc: R.peak_AB(refc, reft)
    else:
        O, kind, cores = Oracle(), "port", 1
        peak_ab = lambda refc: O.ref_peak_AB(refc, reft)
    P = cands.n
    done, t_total, n_steps = 0, 0.0, 0
    idx = 0
    while True:
        for c0 in range(0, per_step, REF_SAMPLE_CANDS):
            m = min(REF_SAMPLE_CANDS, per_step - c0)
            sel = np.arange(idx, idx + m) % P
            idx += m
            refc = reference_candidates(cands.subset(sel))
            t = time.perf_counter()
            A, B = peak_ab(refc)
            h0, dd, dk = A @ w, -(B @ wg), -(A @ wg2)
            t_total += time.perf_counter() - t
            done += m * n_use
        n_steps += 1
        if (steps is not None and n_steps >= steps) or (steps is None and t_total >= seconds):
            break
    return done / t_total, kind, cores, n_steps, t_total


def reference_polish_form(table, cands, k: float, n_use: int) -> dict:
    """The other form of the reference's h0: compute_peak_AB, then polish_peaks_with_weights with
    grid_steps = 0 (path1_eval_fast.cpp:58-143; it returns h0 in out_h_unpol and also runs its
    Newton passes), on one call of REF_SAMPLE_CANDS candidates; zero-terms counted as for the
    NumPy form (candidates x zeros)."""
    from oracle.oracle import RefLib, reference_candidates, reference_format
    if not RefLib.available():
        return {"unavailable": "oracle/_ref/libpath1_eval.so not built"}
    R = RefLib()
    reft = reference_format(table, n_use, exact_psi=False)
    w = np.exp(-k * table.gamma[:n_use] ** 2)
    refc = reference_candidates(cands.subset(np.arange(REF_SAMPLE_CANDS)))
    t = time.perf_counter()
    A, B = R.peak_AB(refc, reft)
    R.polish(A, B, table.gamma[:n_use], w, 0.0, 0)
    secs = time.perf_counter() - t
    return {"value": REF_SAMPLE_CANDS * n_use / secs, "seconds": secs,
            "sample": f"{REF_SAMPLE_CANDS} candidates x {n_use} zeros: compute_peak_AB + "
                      "polish_peaks_with_weights(grid_steps=0), value only"}


def workload_config(world: int, n_T: int) -> dict:
    """The workload both arms run (the same dict in both lines)."""
    return {"workload": WORKLOAD, "zeros": n_T, "candidates_per_gpu": P_PER_GPU, "k": K_GAUSS, "T0": T0,
            "tol": TOL, "l2": "GPU arm: a 256 MB buffer written between timed steps (the 28 MB table "
                              "would otherwise stay in the 126 MB L2)",
            "parallelism": f"candidates sharded over {world} GPU(s), no collective on the data path"}


# ---------------------------------------------------------------- our arm

def run_ours(args):
    import torch
    import torch.distributed as dist
    from mertens_bound_b200 import k2, synth, _lib
    from mertens_bound_b200._lib import check

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local])

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    data = synth.make_table_below(T0, seed=1)
    cands = synth.make_candidates(P_PER_GPU, seed=3 + rank)
    P = cands.n
    table = k2.ZeroTable.from_data(data, device=local)
    n_T = table.count_below(T0)
    terms = float(P) * n_T

    vi = torch.from_numpy(cands.v_int.view(np.int64)).to(dev)
    vf = torch.from_numpy(cands.v_frac.view(np.int64)).to(dev)
    dl = torch.zeros(P, dtype=torch.float64, device=dev)
    out = torch.empty(3, P, dtype=torch.float64, device=dev)
    ref = torch.empty(3, P, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)   # > 126 MB L2
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream
    L = _lib.lib()

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize(dev)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for s in range(steps):
            flush.fill_(s & 0xFF)                # evict table + candidates from L2 between steps
            ev[s][0].record(stream)
            fn()
            ev[s][1].record(stream)
        torch.cuda.synchronize(dev)
        return [a.elapsed_time(b) for a, b in ev]

    # plain FP64 kernel (denominator of the ratio)
    def plain():
        check(L.mb_k2_plain_dev(table.handle, P, vi.data_ptr(), vf.data_ptr(), dl.data_ptr(), K_GAUSS, T0,
                                ref[0].data_ptr(), ref[1].data_ptr(), ref[2].data_ptr(), sptr))
    plain_ms = timed(plain, max(3, args.steps // 10), 2)

    plan = k2.Plan(table, [P], [K_GAUSS], [T0], tol=TOL)
    gi = plan.group_info(0)
    from mertens_bound_b200.autotune import autotune
    t_tune = time.perf_counter()
    tuned = autotune(plan, reps=3, use_cache=False)
    tune_s = time.perf_counter() - t_tune

    def fast(tiers=3):
        check(L.mb_plan_run_tiers_dev(plan.handle, tiers, vi.data_ptr(), vf.data_ptr(), dl.data_ptr(),
                                      out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), sptr))

    # headline: chosen form, exactly K timed steps bracketed by barrier + synchronize; the plan
    # records CUDA events around each step's light and heavy launches (the kernels' own durations
    # inside the concurrent step, on the streams they run on)
    for _ in range(max(3, args.warmup)):
        fast()
    check(L.mb_plan_kernel_timing(plan.handle, args.steps))
    torch.cuda.synchronize(dev)
    barrier()
    torch.cuda.synchronize(dev)
    sampler = ClockSampler(local)
    t_wall = time.perf_counter()
    step_ms = timed(fast, args.steps, 0)
    barrier()
    torch.cuda.synchronize(dev)
    wall_s = time.perf_counter() - t_wall
    clocks = sampler.stop()
    total_ms = max_over_ranks(sum(step_ms))
    value = world * terms * args.steps / (total_ms * 1e-3)
    ms_per_step = total_ms / args.steps
    light_in_step, heavy_in_step = kernel_times(L, plan, args.steps)
    check(L.mb_plan_kernel_timing(plan.handle, 0))
    diff = (out - ref).abs().max(dim=1).values.cpu().numpy()
    # error against rigorous enclosures: the certified interval kernel on a 64-candidate subsample
    # (the error of a value inside nothing wider than the interval is below |val - mid| + width/2)
    sub = cands.subset(np.arange(64))
    clo, chi, _ = k2.k2_certified(table, sub, K_GAUSS, T0)
    got = out[0, :64].cpu().numpy()
    mid, half = 0.5 * (clo + chi), 0.5 * (chi - clo)
    err_vs_cert = float(np.max(np.abs(got - mid) + half))

    # per-tier kernels on their own
    light_ms = statistics.median(timed(lambda: fast(2), 5, 1))
    heavy_ms = statistics.median(timed(lambda: fast(1), 5, 1))
    ht, lt = C_double_pair(L.mb_plan_tier_terms, plan.handle)
    ffma_peak, mufu_peak, dfma_peak = calibrate_pipes(L, local)

    # end to end through the host-pointer API (pinned H2D, graph, D2H), every step
    for _ in range(3):
        plan.run(cands)
    barrier()
    t = time.perf_counter()
    for _ in range(args.steps):
        plan.run(cands)
    e2e_s = max_over_ranks(time.perf_counter() - t)
    e2e_value = world * terms * args.steps / e2e_s

    # the same scoring with the negligible tail skipped (a quarter of tol): not the headline
    # (that evaluates every zero below T0, as the reference does), the time a user gets
    plan.set_skip(0.25)
    gs = plan.group_info(0)
    skip_ms = statistics.median(timed(fast, max(10, args.steps // 10), 3))
    tail_skip = {"ms_per_step": skip_ms, "zeros_evaluated": gs["n_eval"], "zeros_below_T0": gs["n_T"],
                 "err_bound": gs["err_bound"], "candidates_per_s": world * P / (skip_ms * 1e-3),
                 "evaluated_zero_terms_per_s": world * P * gs["n_eval"] / (skip_ms * 1e-3),
                 "speedup_vs_full_step": ms_per_step / skip_ms}
    plan.set_skip(0.0)

    plain_step_ms = statistics.median(plain_ms)
    plain_rate = terms / (plain_step_ms * 1e-3)
    cpt = tuned["config"][0]
    one_kernel = tuned["config"][3] >= 1
    # in-step durations: with one persistent kernel both tiers share one launch (recorded as the
    # light pair of events); otherwise each tier kernel has its own
    light_mean = statistics.fmean(light_in_step)
    heavy_mean = light_mean if one_kernel else statistics.fmean(heavy_in_step)
    mufu_achieved = LIGHT_MUFU_PER_TERM * lt / (light_mean * 1e-3)
    fp64_achieved = HEAVY_FP64_PER_TERM * ht / (heavy_mean * 1e-3)
    # the dominant kernel: the light tier (its work spans most of the step); its binding pipe is
    # XU (two MUFU operations per zero-term), against the XU rate measured live on this GPU
    roofline = {
        "bound": "xu",
        "kernel": ("k2_tiers_kernel (both tiers in one persistent kernel; XU work of its light items)"
                   if one_kernel else "k2_light_kernel (light tier), inside the concurrent step"),
        "achieved": mufu_achieved / 1e12, "peak": mufu_peak / 1e12, "unit": "T MUFU-op/s",
        "frac": mufu_achieved / mufu_peak,
        "traffic": TIERS_DRAM_BYTES if one_kernel else LIGHT_DRAM_BYTES[cpt],
        "traffic_unit": "bytes/launch (ncu dram read+write)",
        "algorithmic": f"{LIGHT_MUFU_PER_TERM} MUFU (sin, cos) per light zero-term",
        "peak_source": "measured live: sin.approx/cos.approx chains (mb_calibrate_pipes)",
        "light_terms": lt, "light_ms_in_step": light_mean,
        "light_alone_ms": light_ms, "light_alone_frac": LIGHT_MUFU_PER_TERM * lt / (light_ms * 1e-3) / mufu_peak,
        "heavy_terms": ht, "heavy_ms_in_step": heavy_mean, "heavy_alone_ms": heavy_ms,
        "heavy_fp64_achieved": fp64_achieved / 1e12, "heavy_fp64_peak": dfma_peak / 1e12,
        "heavy_fp64_frac": fp64_achieved / dfma_peak,
        "heavy_alone_fp64_frac": HEAVY_FP64_PER_TERM * ht / (heavy_ms * 1e-3) / dfma_peak,
        "heavy_traffic": HEAVY_DRAM_BYTES,
        "step_xu_frac": LIGHT_MUFU_PER_TERM * lt / (ms_per_step * 1e-3) / mufu_peak,
        "step_fp64_frac": HEAVY_FP64_PER_TERM * ht / (ms_per_step * 1e-3) / dfma_peak,
        # both tiers' algorithmic work at their pipes' peaks, one after the other, over the step:
        # the fraction of a step whose pipes could not overlap
        "step_pipe_time_frac": (LIGHT_MUFU_PER_TERM * lt / mufu_peak + HEAVY_FP64_PER_TERM * ht / dfma_peak)
                               / (ms_per_step * 1e-3),
        "issue_frac_side": (LIGHT_INST_PER_TERM[cpt] * lt + HEAVY_INST_PER_TERM * ht) / (ms_per_step * 1e-3)
                           / ffma_peak,
        "hbm_frac_side": (LIGHT_DRAM_BYTES[cpt] + HEAVY_DRAM_BYTES) / (ms_per_step * 1e-3) / 1e9 / hbm_peak()[0],
        "plain_fp64_ms_per_step": plain_step_ms, "plain_fp64_value": world * plain_rate,
        "speedup_vs_plain": value / (world * plain_rate),
        "err_bound": gi["err_bound"], "err_bound_dd": gi["err_bound_dd"], "err_bound_dk": gi["err_bound_dk"],
        "err_vs_certified_max": err_vs_cert, "max_abs_diff_vs_plain": float(diff[0]),
        "heavy_zeros": gi["n_heavy"], "light_form": plan.info()["light_form"],
        "tile_light_cpt": cpt, "tile_nzw_shift": tuned["config"][1], "tile_chunk_scale": tuned["config"][2],
        "schedule": {0: "heavy and light tier kernels concurrently", 1: "one persistent kernel, heavy items first",
                     2: "one persistent kernel, items by cost",
                     3: "one persistent kernel, one queue per tier"}[tuned["config"][3]],
    }
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32 phase + f64 (heavy tier) + f32 (light tier)",
        "data": "synthetic (seeded zero table and candidates; no real zeta zeros)",
        "config": workload_config(world, n_T),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 3 * 8 * P, "d2h_bytes_per_step": 3 * 8 * P},
        "roofline": roofline,
        "clocks": clocks,
        "gpu_launches": (2 if one_kernel else 3) * args.steps,
        "wall_s_timed_region": wall_s,
        "accuracy": {"err_vs_certified": {"candidates": 64, "max_abs_err": err_vs_cert,
                                          "max_interval_width": float(np.max(chi - clo)),
                                          "a_priori_bound": gi["err_bound"]},
                     "max_abs_diff_vs_plain": {"val": float(diff[0]), "dd": float(diff[1]), "dk": float(diff[2])}},
        "autotune_s": tune_s,
        "tail_skip": tail_skip,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, kind, cores, calls, secs = reference_rate(data, cands, K_GAUSS, n_T, args.cpu_seconds)
        pf = reference_polish_form(data, cands, K_GAUSS, n_T)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
                                "sample": f"{calls} calls x {REF_SAMPLE_CANDS} candidates x {n_T} zeros "
                                          f"({secs:.1f} s): compute_peak_AB + value/grad sums as NumPy dots",
                                "nproc": os.cpu_count(), "polish_form_value": pf.get("value"),
                                "polish_form_sample": pf.get("sample", pf.get("unavailable"))}
    plan.close()
    table.close()
    if world == 1 and not args.no_workloads:
        line["workloads"] = other_workloads(torch, dev, timed, cpu_baseline=not args.no_cpu_baseline)
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def _ball_chunk(args):
    """One worker's share of the interval restatement (oracle/interval.py) of the certified sum."""
    from oracle.interval import k2_ball
    vi, vf, G3, cre, cim, k = args
    k2_ball(vi, vf, 0.0, G3, cre, cim, k, len(cre))
    return len(cre)


def certified_cpu_rate(big, pk, n_full: int, per_worker: int = 1500):
    """Zeros/s of the certified sum on the host cores: the 220-bit interval restatement of
    certify_K2.work (python-flint, the reference's ball library, is not installed), one chunk of
    per_worker zeros per core spread over the table, in a spawn pool (the GPU is already in use)."""
    import multiprocessing as mp
    n = os.cpu_count() or 1
    starts = np.linspace(0, big.n - per_worker, n).astype(int)
    tasks = [(int(pk.v_int[0]), int(pk.v_frac[0]), big.G3[a:a + per_worker].copy(), big.c_re[a:a + per_worker].copy(),
              big.c_im[a:a + per_worker].copy(), 1.5e-10) for a in starts]
    try:
        with mp.get_context("spawn").Pool(n) as pool:
            warm = [(a, b, G[:16], c, d, k) for a, b, G, c, d, k in tasks]
            pool.map_async(_ball_chunk, [(a, b, G, c[:16], d[:16], k) for a, b, G, c, d, k in warm],
                           chunksize=1).get(timeout=300)         # imports
            t0 = time.perf_counter()
            done = sum(pool.map_async(_ball_chunk, tasks, chunksize=1).get(timeout=600))
            secs = time.perf_counter() - t0
    except Exception as e:                                       # a worker failed or timed out
        return {"kind": "port", "unavailable": f"{type(e).__name__}: {e}"}
    rate = done / secs
    return {"kind": "port", "cores": n, "zeros_per_s": rate, "full_sum_s_extrapolated": n_full / rate,
            "sample": f"{done} zeros ({n} chunks of {per_worker} spread over the table), mpmath iv at 220 bits "
                      "restating certify_K2.work; python-flint is not installed"}


_HP = {}


def _hp_init(ta, gamma):
    _HP["ta"], _HP["gamma"] = ta, gamma


def _hp_one(top):
    """One hit through the restated ZeroData::polish, all five stages (no early exit)."""
    from oracle.oracle import zerodata_polish
    zerodata_polish(top, _HP["ta"], _HP["gamma"], thresholds=(None, None, None))
    return 1


def _hp_warm(_):
    import oracle.oracle  # noqa: F401
    return 0


def screen_cpu(reft, two_astar, pts):
    """Leaves/s of the enumerators' CPU screen ZeroData::fast_screen (C restatement in the oracle,
    OpenMP over leaves on all host cores as the enumerator runs it) on the same leaves; x =
    floor(v 2^30) as the enumerators hold them."""
    from oracle.oracle import Oracle
    vi, vf = pts[:, 0].astype(np.uint64), pts[:, 1].astype(np.uint64)
    x_lo = (vi << np.uint64(30)) | (vf >> np.uint64(34))
    x_hi = vi >> np.uint64(34)
    O = Oracle()
    O.fast_screen(x_lo[:4096], x_hi[:4096], reft, two_astar)
    t0 = time.perf_counter()
    flags = O.fast_screen(x_lo, x_hi, reft, two_astar)
    secs = time.perf_counter() - t0
    return {"kind": "port", "cores": os.cpu_count(), "leaves": int(len(x_lo)), "seconds": secs,
            "leaves_per_s": len(x_lo) / secs, "passed": int(flags.sum()),
            "sample": "all leaves; ZeroData::fast_screen restated in C (64 + 64 zeros, 14-bit FP32 cosine "
                      "table, 7 offsets, thresholds 0.810 / 0.875)"}


def hit_polish_cpu(d600, hits, reft):
    """Hits/s of ZeroData::polish on the host cores: the numpy restatement of
    search/gpu_mertens_stream.cu:381-505 (all five stages, every hit to the end), one hit per core
    in a spawn pool; the reference runs the same stages in C++ with OpenMP over hits.  The hits'
    phase words come from the restated compute_peak_AB on the reference's table layout."""
    import multiprocessing as mp
    from oracle.oracle import MASK64, Oracle
    n = os.cpu_count() or 1
    x = [(int(a) << 30) | (int(b) >> 34) for a, b in hits[:n]]
    x_lo = np.array([v & MASK64 for v in x], np.uint64)
    x_hi = np.array([v >> 64 for v in x], np.uint64)
    _, _, top = Oracle().ref_peak_AB((x_lo, x_hi, np.zeros(len(x))), reft, want_top=True)
    ta = 2.0 * reft["alpha"] * np.exp(-3e-9 * d600.gamma ** 2)
    try:
        with mp.get_context("spawn").Pool(n, initializer=_hp_init, initargs=(ta, d600.gamma)) as pool:
            pool.map_async(_hp_warm, range(n), chunksize=1).get(timeout=300)
            t0 = time.perf_counter()
            done = sum(pool.map_async(_hp_one, [row.view(np.int64) for row in top], chunksize=1).get(timeout=600))
            secs = time.perf_counter() - t0
    except Exception as e:                                       # a worker failed or timed out
        return {"kind": "port", "unavailable": f"{type(e).__name__}: {e}"}
    return {"kind": "port", "cores": n, "hits": done, "seconds": secs, "hits_per_s": done / secs,
            "sample": f"{done} of the same hits, one per core; numpy restatement of ZeroData::polish "
                      "(oracle.zerodata_polish), phase words from the restated compute_peak_AB"}


def polish_scan_cpu(t74, n74, m_half: int = 200):
    """Point-zero terms/s of search/polish.py's FP64 grid (oracle.polish_ref.scan_grid: angles
    phi + m dphi, cos and sin per term, numpy on one core as in the reference) on 2 m_half points of
    the same scan; phi and dphi are the exact phases (polish.py reduces them with mpfr, untimed
    here as there)."""
    from fractions import Fraction
    from mertens_bound_b200 import polish, synth
    from oracle.oracle import Oracle
    from oracle.polish_ref import scan_grid
    O = Oracle()
    G3 = t74.G3[:n74]
    vi, vf = polish.to_fixed(synth.PEAK2_STR)
    si, sf = polish.to_fixed(Fraction(2e-5))
    two_pi = 2.0 * math.pi
    ph = O.phase128(synth.Candidates(np.array([vi], np.uint64), np.array([vf], np.uint64), np.zeros(1)), G3, n74)[0]
    dp = O.phase128(synth.Candidates(np.array([si], np.uint64), np.array([sf], np.uint64), np.zeros(1)), G3, n74)[0]
    phi = ph[0].astype(np.float64) * (two_pi / 2.0 ** 64)
    dphi = dp[0].astype(np.float64) * (two_pi / 2.0 ** 64)
    w = np.exp(-3e-9 * t74.gamma[:n74] ** 2)
    gre, gim = w * t74.c_re[:n74], w * t74.c_im[:n74]
    t0 = time.perf_counter()
    scan_grid(phi, dphi, gre, gim, -m_half, m_half, chunk=2 * m_half)
    secs = time.perf_counter() - t0
    terms = 2 * m_half * n74
    return {"kind": "port", "cores": 1, "points": 2 * m_half, "seconds": secs,
            "point_zero_terms_per_s": terms / secs,
            "sample": f"{2 * m_half} of the 25,001 grid points over all {n74} zeros, one chunk "
                      "(polish.py uses chunks of 4,000 points)"}


def other_workloads(torch, dev, timed, cpu_baseline: bool = True):
    """The other four workload shapes, measured briefly on the same GPU (summary numbers)."""
    from mertens_bound_b200 import k2, synth, _lib
    from mertens_bound_b200._lib import check
    from mertens_bound_b200.autotune import autotune
    L = _lib.lib()
    sptr = torch.cuda.current_stream(dev).cuda_stream
    out = {}

    def dev_cands(c):
        return (torch.from_numpy(c.v_int.view(np.int64).copy()).to(dev),
                torch.from_numpy(c.v_frac.view(np.int64).copy()).to(dev),
                torch.from_numpy(c.delta.copy()).to(dev))

    def plain_run(t, vi, vf, dl, o, k, T, off=0, n=None):
        n = vi.shape[0] if n is None else n
        check(L.mb_k2_plain_dev(t.handle, n, vi[off:].data_ptr(), vf[off:].data_ptr(), dl[off:].data_ptr(), k, T,
                                o[0, off:].data_ptr(), o[1, off:].data_ptr(), o[2, off:].data_ptr(), sptr))

    def plan_run(plan, vi, vf, dl, o):
        plan.run_dev(vi.data_ptr(), vf.data_ptr(), dl.data_ptr(), o[0].data_ptr(), o[1].data_ptr(),
                     o[2].data_ptr(), sptr)

    # small_plain: 64 candidates x 10,000 zeros, k = 3e-9
    small = synth.make_table(10_000, seed=1)
    c1 = synth.make_candidates(64, seed=2)
    with k2.ZeroTable.from_data(small, device=dev.index) as t:
        vi, vf, dl = dev_cands(c1)
        o1 = torch.empty(3, 64, dtype=torch.float64, device=dev)
        o2 = torch.empty_like(o1)
        pm = statistics.median(timed(lambda: plain_run(t, vi, vf, dl, o1, 3e-9, math.inf), 20, 3))
        with k2.Plan(t, [64], [3e-9], [math.inf], tol=TOL) as plan:
            autotune(plan, reps=3, use_cache=False)
            fm = statistics.median(timed(lambda: plan_run(plan, vi, vf, dl, o2), 20, 3))
            eb = plan.group_info(0)["err_bound"]
        terms = 64 * 10_000
        out["small_plain"] = {"zero_terms": terms, "plain_ms": pm, "chosen_ms": fm,
                              "plain_rate": terms / pm * 1e3, "chosen_rate": terms / fm * 1e3,
                              "max_abs_diff": float((o2[0] - o1[0]).abs().max()), "err_bound": eb}

    big = synth.make_table(2_325_572, seed=1)
    with k2.ZeroTable.from_data(big, device=dev.index) as tb:
        # certified_full: Peak2, all 2,325,572 zeros below 1.3e6, k = 1.5e-10
        pk = synth.peak2_candidate()
        k2.k2_certified(tb, pk, 1.5e-10, 1.3e6, v_rad=2.0 ** -64)
        ts = []
        for _ in range(5):
            t0 = time.perf_counter()
            lo, hi, ab = k2.k2_certified(tb, pk, 1.5e-10, 1.3e6, v_rad=2.0 ** -64)
            ts.append(time.perf_counter() - t0)
        out["certified_full"] = {"zeros": tb.count_below(1.3e6), "seconds": statistics.median(ts),
                                 "lo": float(lo[0]), "hi": float(hi[0]), "width": float(hi[0] - lo[0]),
                                 "abs_sum_hi": float(ab[0])}
        if cpu_baseline:
            out["certified_full"]["cpu_baseline"] = certified_cpu_rate(big, pk, out["certified_full"]["zeros"])

        # batched_uneven: 16,384 candidates in 12 groups over T x k
        counts, ks, Ts = synth.batched_uneven_groups()
        c4 = synth.make_candidates(sum(counts), seed=4)
        vi, vf, dl = dev_cands(c4)
        o1 = torch.empty(3, c4.n, dtype=torch.float64, device=dev)
        o2 = torch.empty_like(o1)
        with k2.Plan(tb, counts, ks, Ts, tol=TOL) as plan:
            tuned = autotune(plan, reps=2, use_cache=False)
            fm = statistics.median(timed(lambda: plan_run(plan, vi, vf, dl, o2), 5, 2))
            terms = plan.info()["zero_terms"]
            bounds = [plan.group_info(g)["err_bound"] for g in range(len(counts))]

            def plain_all():
                off = 0
                for c, k, T in zip(counts, ks, Ts):
                    plain_run(tb, vi, vf, dl, o1, k, T, off, c)
                    off += c
            pm = statistics.median(timed(plain_all, 3, 1))
        out["batched_uneven"] = {"zero_terms": terms, "groups": len(counts), "chosen_ms": fm, "plain_ms": pm,
                                 "chosen_rate": terms / fm * 1e3, "plain_rate": terms / pm * 1e3,
                                 "speedup_vs_plain": pm / fm, "max_abs_diff": float((o2[0] - o1[0]).abs().max()),
                                 "max_err_bound": max(bounds), "autotuned": list(tuned["config"])}

        # newton_polish: 1,024 candidates, T0 = 1.3e6, k = 1.5e-10, 8 Newton steps
        c5 = synth.make_candidates(1024, seed=5)
        vi, vf, dl = dev_cands(c5)
        o2 = torch.empty(3, 1024, dtype=torch.float64, device=dev)
        with k2.Plan(tb, [1024], [1.5e-10], [1.3e6], tol=TOL) as plan:
            autotune(plan, reps=3, use_cache=False)
            em = statistics.median(timed(lambda: plan_run(plan, vi, vf, dl, o2), 5, 2))
            h4 = torch.empty(4, 1024, dtype=torch.float64, device=dev)
            d = dl.clone()

            def newton():
                d.copy_(dl)
                check(L.mb_plan_newton_dev(plan.handle, vi.data_ptr(), vf.data_ptr(), d.data_ptr(), 8, 1e-4,
                                           h4[0].data_ptr(), h4[1].data_ptr(), h4[2].data_ptr(), h4[3].data_ptr(),
                                           sptr))
            nm = statistics.median(timed(newton, 3, 1))
            terms = 1024.0 * tb.count_below(1.3e6)
            gain = float((h4[1].abs() - h4[0].abs()).mean())
        out["newton_polish"] = {"zero_terms_per_eval": terms, "eval_ms": em, "eval_rate": terms / em * 1e3,
                                "newton8_ms": nm, "evals_per_newton": 10, "mean_abs_gain": gain}

    # driver_scoring: the search drivers' step (search/eval_tech1_600k.py:216-273) -- 256
    # candidates over the first 600,000 zeros, polish_peaks_with_weights under the five weight
    # vectors -- matrix-free on the GPU; beside it the reference's compiled evaluator
    # (compute_peak_AB once + five polishes) on 16 of the candidates
    from mertens_bound_b200 import score
    d600 = big.truncate(600_000)
    c6 = synth.make_candidates(256, seed=6)
    c6.delta[:] = np.random.default_rng(6).uniform(-1e-4, 1e-4, 256)
    W = score.reference_weights(d600.gamma)
    with k2.ZeroTable.from_data(d600, device=dev.index) as t6:
        slots = score.register(t6, W)                                    # once per table
        score.score(t6, c6.subset(np.arange(8)), slots)
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            res = score.score(t6, c6, slots)
            ts.append(time.perf_counter() - t0)
        gpu_s = statistics.median(ts)
    ds = {"candidates": 256, "zeros": 600_000, "weights": list(W), "grid": "2.5e-4 / 40 steps",
          "seconds": gpu_s, "candidates_per_s": 256 / gpu_s, "timing": "median of 3 calls, slots registered once",
          "best_abs_h_pol": float(max(np.max(np.abs(v[1])) for v in res.values()))}
    if cpu_baseline:
        try:
            from oracle.oracle import RefLib, reference_candidates, reference_format
            if RefLib.available():
                R = RefLib()
                sub = c6.subset(np.arange(16))
                reft = reference_format(d600, exact_psi=False)
                t0 = time.perf_counter()
                A, B = R.peak_AB(reference_candidates(sub), reft)
                for w in W.values():
                    R.polish(A, B, d600.gamma, w, 2.5e-4, 40)
                cs = time.perf_counter() - t0
                ds["cpu_baseline"] = {"kind": "reference", "cores": 16, "candidates": 16, "seconds": cs,
                                      "candidates_per_s": 16 / cs,
                                      "sample": "compute_peak_AB + 5 x polish_peaks_with_weights, "
                                                "search/path1_eval_fast.cpp compiled in oracle/_ref"}
        except Exception as e:                                       # the baseline is optional
            ds["cpu_baseline"] = {"unavailable": f"{type(e).__name__}: {e}"}
    out["driver_scoring"] = ds

    # driver_dropin: the same step with the drivers unchanged, through the library's
    # compute_peak_AB / polish_peaks_with_weights (search/eval_tech1_600k.py:216-273 calling
    # libmertens_k2.so in place of libpath1_eval.so): the A and B matrices of 64 candidates
    # (2 x 307 MB) come to the host once and go back to the device for each of the five polishes
    from mertens_bound_b200 import compat, formats
    f6 = formats.reference_fields(d600, exact_psi=False)
    sub = c6.subset(np.arange(64))
    xs = [(int(a) << 30) | (int(b) >> 34) for a, b in zip(sub.v_int, sub.v_frac)]
    x_lo = np.array([v & 0xFFFFFFFFFFFFFFFF for v in xs], np.uint64)
    x_hi = np.array([v >> 64 for v in xs], np.uint64)
    dy0 = np.array([int(b) & ((1 << 34) - 1) for b in sub.v_frac], dtype=np.float64) * 2.0 ** -64 + sub.delta

    def dropin():
        A, B = compat.compute_peak_AB(x_lo, x_hi, dy0, f6["alpha"], f6["gamma"], f6["ghi_lo"], f6["ghi_hi"],
                                      f6["glo_lo"], f6["glo_hi"], f6["psi_lo"], f6["psi_hi"])
        return [compat.polish_peaks_with_weights(A, B, d600.gamma, w, 2.5e-4, 40) for w in W.values()]
    dropin()
    t0 = time.perf_counter()
    dropin()
    di_s = time.perf_counter() - t0
    out["driver_dropin"] = {"candidates": 64, "zeros": 600_000, "seconds": di_s, "candidates_per_s": 64 / di_s,
                            "note": "unchanged drivers through the compute_peak_AB / polish_peaks_with_weights "
                                    "exports: host A/B matrices cross PCIe once out and five times in"}

    # the enumerators' two GPU steps and the peak re-optimisation, each on the 600,000-zero table:
    #   enumerator_screen  2^20 random leaves through the GPU screen (64/128/256 zeros, 7 offsets)
    #   hit_polish         256 hits through the five ZeroData::polish stages
    #   polish_scan        search/polish.py's default grid (half 0.25, step 2e-5: 25,001 points) over
    #                      the zeros below 74,000 at the Peak2 point
    from mertens_bound_b200 import hit_polish, path1, polish
    with k2.ZeroTable.from_data(d600, device=dev.index) as t6:
        cl = synth.make_candidates(1 << 20, seed=7)
        pts = np.stack([cl.v_int, cl.v_frac], axis=1)
        hit_polish.screen_leaves(t6, pts[:4096])

        def wall(fn, reps=3):
            """Median wall seconds of fn() over reps calls, and its last result."""
            ts = []
            for _ in range(reps):
                t0 = time.perf_counter()
                res = fn()
                ts.append(time.perf_counter() - t0)
            return statistics.median(ts), res

        sc_s, r = wall(lambda: hit_polish.screen_leaves(t6, pts, max_hits=1 << 20))
        out["enumerator_screen"] = {"leaves": len(pts), "seconds": sc_s, "leaves_per_s": len(pts) / sc_s,
                                    "hits": int(len(r.hits)), "stages": "64/128/256 zeros, 0.78/0.855/0.892",
                                    "note": "host-pointer call: includes the H2D of 16 MB of leaves; median of 3 calls"}
        # the same screen on leaves already in HBM (mb_screen_dev), device-timed
        dvi = torch.from_numpy(pts[:, 0].view(np.int64).copy()).to(dev)
        dvf = torch.from_numpy(pts[:, 1].view(np.int64).copy()).to(dev)
        cap = 1 << 16
        dh = torch.empty(cap, dtype=torch.int64, device=dev)
        dhs = torch.empty(cap, 3, dtype=torch.float32, device=dev)
        dn = torch.empty(1, dtype=torch.int64, device=dev)

        def screen_dev():
            hit_polish.screen_leaves_dev(t6, dvi.data_ptr(), dvf.data_ptr(), len(pts), dh.data_ptr(),
                                         dhs.data_ptr(), dn.data_ptr(), cap, stream=sptr)
        ds = statistics.median(timed(screen_dev, 5, 2)) * 1e-3
        out["enumerator_screen"].update({"device_seconds": ds, "device_leaves_per_s": len(pts) / ds,
                                         "device_note": "mb_screen_dev on leaves in HBM, CUDA events, median of 5"})
        reft = None
        if cpu_baseline:
            try:
                from oracle.oracle import reference_format
                reft = reference_format(d600, exact_psi=False)
                ta600 = 2.0 * reft["alpha"] * np.exp(-3e-9 * d600.gamma ** 2)
                out["enumerator_screen"]["cpu_baseline"] = screen_cpu(reft, ta600, pts)
            except Exception as e:                                   # the baseline is optional
                out["enumerator_screen"]["cpu_baseline"] = {"unavailable": f"{type(e).__name__}: {e}"}
        hits = pts[:256]
        hit_polish.polish_hits(t6, hits[:8])
        hp_s, hr = wall(lambda: hit_polish.polish_hits(t6, hits, thresholds=(None, None, None)))
        out["hit_polish"] = {"hits": 256, "zeros": d600.n, "seconds": hp_s, "hits_per_s": 256 / hp_s,
                             "stages_run": int(hr.stage.max()) + 1, "thresholds": "none (every hit runs all stages)"}
        if reft is not None:
            out["hit_polish"]["cpu_baseline"] = hit_polish_cpu(d600, hits, reft)
        n74 = t6.count_below(polish.POLISH_T)
        polish.scan(t6, synth.PEAK2_STR, 0.001, 2e-5)
        ps_s, (best, y_best, m_best) = wall(lambda: polish.scan(t6, synth.PEAK2_STR, 0.25, 2e-5))
        out["polish_scan"] = {"points": 25001, "zeros": n74, "seconds": ps_s,
                              "point_zero_terms_per_s": 25001 * n74 / ps_s, "best_abs_h": abs(best)}
        if cpu_baseline:
            try:
                out["polish_scan"]["cpu_baseline"] = polish_scan_cpu(d600, n74)
            except Exception as e:                                   # the baseline is optional
                out["polish_scan"]["cpu_baseline"] = {"unavailable": f"{type(e).__name__}: {e}"}

    # taylor_polish: search/path1_kernel_opt.py's fast_polish_batch_blas contract (degree-16
    # moments, 121-point grid, exact Newton on the top 25) for 1,024 candidates over its 100,000
    # zeros with the JP weight, matrix-free; beside it the reference algorithm (numpy/BLAS
    # restatement) on A/B rows from the reference's compiled compute_peak_AB
    d100 = big.truncate(100_000)
    c7 = synth.make_candidates(1024, seed=8)
    w_jp = score.reference_weights(d100.gamma)["jp"]
    with k2.ZeroTable.from_data(d100, device=dev.index) as t7:
        slot = t7.add_weights(w_jp)
        path1.fast_polish_exact(t7, c7.subset(np.arange(64)), slot)
        t0 = time.perf_counter()
        path1.fast_polish_exact(t7, c7, slot)
        tp_s = time.perf_counter() - t0
    tp = {"candidates": 1024, "zeros": 100_000, "seconds": tp_s, "candidates_per_s": 1024 / tp_s,
          "top": 25, "grid": "121 points on [-3e-5, 3e-5]"}
    if cpu_baseline:
        try:
            from oracle import polish_ref
            from oracle.oracle import RefLib, reference_candidates, reference_format
            if RefLib.available():
                sub = c7.subset(np.arange(128))
                A, B = RefLib().peak_AB(reference_candidates(sub), reference_format(d100, exact_psi=False))
                t0 = time.perf_counter()
                polish_ref.fast_polish_batch(A, B, d100.gamma, w_jp)
                cs = time.perf_counter() - t0
                tp["cpu_baseline"] = {"kind": "port", "cores": os.cpu_count(), "candidates": 128, "seconds": cs,
                                      "candidates_per_s": 128 / cs,
                                      "sample": "numpy/BLAS restatement of fast_polish_batch_blas on A/B rows "
                                                "(A/B build not timed)"}
        except Exception as e:
            tp["cpu_baseline"] = {"unavailable": f"{type(e).__name__}: {e}"}
    out["taylor_polish"] = tp
    return out


def C_double(fn, *args):
    import ctypes as C
    from mertens_bound_b200._lib import check
    x = C.c_double()
    check(fn(*args, C.byref(x)))
    return x.value


def C_double_pair(fn, *args):
    import ctypes as C
    from mertens_bound_b200._lib import check
    a, b = C.c_double(), C.c_double()
    check(fn(*args, C.byref(a), C.byref(b)))
    return a.value, b.value


def kernel_times(L, plan, n: int):
    """The light and heavy kernel durations (ms) of the plan's last n timed runs."""
    import ctypes as C
    from mertens_bound_b200._lib import check
    lt, ht, got = (C.c_double * n)(), (C.c_double * n)(), C.c_int()
    check(L.mb_plan_kernel_times(plan.handle, n, lt, ht, C.byref(got)))
    if got.value != n:
        raise RuntimeError(f"kernel timing recorded {got.value} of {n} runs")
    return list(lt), list(ht)


def calibrate_pipes(L, device: int):
    """Measured FFMA, MUFU and DFMA thread-op rates of this GPU (ops/s)."""
    import ctypes as C
    from mertens_bound_b200._lib import check
    f, m, d = C.c_double(), C.c_double(), C.c_double()
    check(L.mb_calibrate_pipes(device, C.byref(f), C.byref(m), C.byref(d)))
    return f.value, m.value, d.value


def hbm_peak():
    """The measured HBM copy peak (GB/s) if MEASURED_PEAKS.json holds one, else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError, TypeError):
        return 6650.0, "fallback"


# ---------------------------------------------------------------- reference arm

def run_reference(args):
    """The reference's own evaluator on the same workload: every timed step scores all 4,096
    candidates over the 466,659 zeros (compute_peak_AB in calls of 64 candidates plus the value and
    gradient sums) -- fewer, in whole calls, when K such steps would take longer than
    REF_TIMED_BUDGET_S at the warm-up rate (about 8 s a step on 16 cores); each untimed warm-up
    step is one such call."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from mertens_bound_b200 import synth
    data = synth.make_table_below(T0, seed=1)
    cands = synth.make_candidates(P_PER_GPU, seed=3)
    n_T = data.count_below(T0)
    warm_rate = reference_rate(data, cands, K_GAUSS, n_T, 0.0, steps=max(1, args.warmup))[0]   # warm-up
    # every timed step scores all candidates when K steps fit in REF_TIMED_BUDGET_S at the warm-up
    # rate; otherwise a step is the largest whole number of 64-candidate calls that fits
    per_step = int(REF_TIMED_BUDGET_S * warm_rate / (max(1, args.steps) * n_T))
    per_step = max(REF_SAMPLE_CANDS, min(P_PER_GPU, per_step // REF_SAMPLE_CANDS * REF_SAMPLE_CANDS))
    rate, kind, cores, n_steps, secs = reference_rate(data, cands, K_GAUSS, n_T, 0.0, steps=args.steps,
                                                      per_step=per_step)
    pf = reference_polish_form(data, cands, K_GAUSS, n_T)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / n_steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded zero table and candidates; no real zeta zeros)",
        "config": workload_config(world, n_T),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"every step: {per_step} of the {P_PER_GPU} candidates x {n_T} zeros "
                                   f"in calls of {REF_SAMPLE_CANDS} (compute_peak_AB + value/grad sums as "
                                   f"NumPy dots)",
                         "nproc": os.cpu_count(), "polish_form_value": pf.get("value"),
                         "polish_form_sample": pf.get("sample", pf.get("unavailable"))},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_profile_extras():
    """One launch each of the kernels beside the tiers, at modest sizes (~0.5 GB on the device):
    the certified interval over all 2,325,572 zeros at the Peak2 point, the leaf screen (4,096
    leaves, 64/128/256 zeros), polish_peaks_with_weights matrix-free (32 candidates x 100,000
    zeros), the Taylor-moment polish matrix-free (256 candidates x 100,000 zeros), then the hit
    scans of 16 hits through the five ZeroData::polish stages, polish.py's 25,001-point grid over
    the zeros below 74,000, and the five-weight scoring of 32 candidates from one exact A/B
    matrix (100,000 zeros)."""
    from mertens_bound_b200 import hit_polish, k2, path1, polish, score, synth
    big = synth.make_table(2_325_572, seed=1)
    with k2.ZeroTable.from_data(big) as tb:
        k2.k2_certified(tb, synth.peak2_candidate(), 1.5e-10, 1.3e6, v_rad=2.0 ** -64)
    d = big.truncate(100_000)
    c = synth.make_candidates(4096, seed=9)
    with k2.ZeroTable.from_data(d) as t:
        pts = np.stack([c.v_int, c.v_frac], axis=1)
        r = hit_polish.screen_leaves(t, pts, 3e-9, hit_polish.SCREEN_GPU)
        slot = t.add_weights(np.exp(-3e-9 * d.gamma * d.gamma))
        path1.polish_peaks_exact(t, c.subset(np.arange(32)), slot)
        path1.fast_polish_exact(t, c.subset(np.arange(256)), slot)
        hit_polish.polish_hits(t, pts[:16], thresholds=(None, None, None))
        polish.scan(t, synth.PEAK2_STR, 0.25, 2e-5)
        score.score(t, c.subset(np.arange(32)), score.reference_weights(d.gamma))
    print(json.dumps({"profile_case": "extras", "screen_hits": int(len(r.hits))}), flush=True)


def run_profile_scoring():
    """The drivers' scoring at a capture-sized scale: 64 candidates over 600,000 zeros under the JP
    weight, mb_polish_peaks_weights twice (an exact_ab_kernel and one A/B-matrix polish each;
    ~0.7 GB on the device)."""
    from mertens_bound_b200 import k2, path1, score, synth
    d = synth.make_table(600_000, seed=1)
    c = synth.make_candidates(64, seed=6)
    c.delta[:] = np.random.default_rng(6).uniform(-1e-4, 1e-4, 64)
    with k2.ZeroTable.from_data(d) as t:
        s = t.add_weights(score.reference_weights(d.gamma)["jp"])
        for _ in range(2):
            r = path1.polish_peaks_weights(t, c, [s])
    print(json.dumps({"profile_case": "scoring", "h_pol0": float(r[1][0][0])}), flush=True)


def run_profile_case(args):
    """Fixed cases for ncu captures (no timing, no bench line).
      small   zeros below 1e5, 2,048 candidates: the chosen form (light tier at 4 candidates per
              thread) args.warmup + args.steps times as two concurrent kernels, once as one
              persistent kernel with one queue per tier, then the plain kernel once (~40 MB on
              the device);
      search  the bench workload (zeros below 3e5, 4,096 candidates): the plain kernel once, the
              light tier alone at 2, 3 and 4 candidates per thread, the heavy tier alone, then both
              tiers in one persistent kernel at 4 candidates per thread (~80 MB)."""
    if args.profile_case == "extras":
        return run_profile_extras()
    if args.profile_case == "scoring":
        return run_profile_scoring()
    import torch
    from mertens_bound_b200 import k2, synth, _lib
    from mertens_bound_b200._lib import check

    dev = torch.device("cuda", 0)
    T, P = (1e5, 2048) if args.profile_case == "small" else (T0, P_PER_GPU)
    data = synth.make_table_below(T, seed=1)
    cands = synth.make_candidates(P, seed=3)
    table = k2.ZeroTable.from_data(data)
    vi = torch.from_numpy(cands.v_int.view(np.int64)).to(dev)
    vf = torch.from_numpy(cands.v_frac.view(np.int64)).to(dev)
    dl = torch.zeros(P, dtype=torch.float64, device=dev)
    out = torch.empty(3, P, dtype=torch.float64, device=dev)
    sptr = torch.cuda.current_stream(dev).cuda_stream
    L = _lib.lib()
    plan = k2.Plan(table, [P], [K_GAUSS], [T], tol=TOL)

    def tiers(n):
        check(L.mb_plan_run_tiers_dev(plan.handle, n, vi.data_ptr(), vf.data_ptr(), dl.data_ptr(),
                                      out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), sptr))

    def plain():
        check(L.mb_k2_plain_dev(table.handle, P, vi.data_ptr(), vf.data_ptr(), dl.data_ptr(), K_GAUSS, T,
                                out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), sptr))

    if args.profile_case == "small":
        plan.configure(4, 0, 1.0)
        for _ in range(args.warmup + args.steps):
            tiers(3)
        plan.set_schedule(3)          # both tiers in one persistent kernel, one queue per tier
        tiers(3)
        plain()
    else:
        plain()
        for cpt in (2, 3, 4):
            plan.configure(cpt, 0, 1.0)
            tiers(2)
        tiers(1)
        plan.set_schedule(1)          # both tiers in one persistent kernel (k2_tiers_kernel)
        tiers(3)
    torch.cuda.synchronize(dev)
    ht, lt = C_double_pair(L.mb_plan_tier_terms, plan.handle)
    print(json.dumps({"profile_case": args.profile_case, "zeros": table.count_below(T), "candidates": P,
                      "heavy_terms": ht, "light_terms": lt}), flush=True)
    plan.close()
    table.close()


def main():
    args = parse()
    if args.profile_case:
        run_profile_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
