// Work description of the chosen-form kernel (shared by k2_fast.cu and k2_plan.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "k2_internal.h"

namespace mb {

// One group: a contiguous candidate range evaluated at one (k, T).
struct FastGroup {
    int64_t c0, nc;    // candidates [c0, c0 + nc)
    double k;
    int64_t pbase;     // offset (in doubles) of this group's partial sums
    int n_chunks;      // zero chunks (heavy then light); partial[pbase + (chunk*nc + p-c0)*3 + q]
    int pad;
    const double *w;   // per-zero weights (device) replacing exp(-k gamma^2), or null
};

// One work item: a candidate tile of one group against one zero chunk of one tier.
struct FastItem {
    int64_t c0;        // first candidate (global index)
    int64_t z0, z1;    // zeros [z0, z1)
    int64_t pbase;     // group.pbase + chunk * group.nc * 3
    int nc;            // candidates in this tile
    int group;
    int tier;          // 0 heavy (FP64), 1 light (FP32 + MUFU)
    int cpt;           // candidates per thread: 1, 2 or 4
    int nzw;           // warps splitting the zeros of one candidate set: 1..8
    int pad;
};

constexpr int HEAVY_CPT = 4;     // candidates per thread in the heavy kernel
constexpr int TIERS_COUNTERS = 2 + 256;   // item counters of one launch: two queues + per-SM arrivals

// Device side of a plan: items[0, n_heavy) are heavy-tier items (pulled by the persistent
// heavy kernel), items[n_heavy, n_heavy + n_light) light-tier items (one CTA each).
struct FastPlanDev {
    FastItem *items = nullptr;      // heavy items, then light items
    FastItem *items_one = nullptr;  // the one-kernel schedules' list (items, or a cost-ordered copy)
    FastGroup *groups = nullptr;
    int n_heavy = 0, n_light = 0, n_groups = 0;
    int light_cpt = 4;          // candidates per thread of the light kernel: 2, 3 or 4
    bool fused_phase = false;   // light tier on light_phase32_fused: every zero has gamma below
                                // FUSED_PHASE_GAMMA, so G's integer part is below 2^19
    bool one_kernel = false;    // both tiers in k2_tiers_kernel (one persistent kernel over
                                // items_one) instead of the heavy kernel on a side stream beside
                                // the light kernel
    bool paired = false;        // one_kernel with per-SM roles: one heavy CTA beside one light CTA
    unsigned heavy_grid = 0;    // CTAs of the heavy kernel
    unsigned tiers_grid = 0;    // CTAs of k2_tiers_kernel
    int *counter = nullptr;     // TIERS_COUNTERS item counters
    double *partial = nullptr;
    size_t partial_bytes = 0;   // size of `partial` (a one-tier run clears it first)
};

// Per-term worst-case absolute error of cos/sin (times amplitude) in each tier, per unit of
// amplitude a_j = 2|c_j| w_j:
//   light: __sinf / __cosf on [-pi, pi] (documented 2^-21.41 / 2^-21.19, so 4.2e-7, their
//          internal argument scaling included) + the angle (int->float 2^-26 turn =
//          9.4e-8 rad, the FMUL's rounding 2^-23 rad, fl_down(2pi) 4.8e-8 relative = 1.5e-7 rad)
//          + phase 4.5 2^-32 turn (2.4 with light_phase32_fused; 7e-9 rad): 7.9e-7 in cos / sin;
//          + amplitude and FFMA roundings (2 2^-24) + FP32 summation over a 32-term flush window
//          (31 2^-24): 1.97e-6  ->  2.76e-6, held at 2.8e-6.  (A 16-term window gives 1.80e-6
//          and ~1,000 fewer heavy zeros at the bench workload, but its flush conversions cost
//          more XU time than those zeros: the step measured 1.4% longer.)
//   heavy: phase 2^-48 turn (2.2e-14 rad; the table index and remainder are exact functions
//          of the FP64 phase sum's bits), 2048-entry table + polynomials (cos 3.96e-14, sin
//          7e-17), FP64 roundings  ->  ~7e-14, held at 2e-13 (loose: the heavy amplitude sum is
//          O(1), so this share of the bound is negligible)
constexpr double EPS_LIGHT = 2.8e-6;
// 2 pi (2^19 - 1): below it G = gamma / 2pi has an integer part below 2^19
constexpr double FUSED_PHASE_GAMMA = 6.283185307179586 * 524287.0;
constexpr double EPS_HEAVY = 2.0e-13;

// CUDA events recorded around the tier launches of one run (the per-kernel timing hook of
// mb_plan_kernel_timing): light0/light1 on the launching stream, heavy0/heavy1 on the stream the
// heavy tier runs on.
struct TierEvents {
    cudaEvent_t light0 = nullptr, light1 = nullptr, heavy0 = nullptr, heavy1 = nullptr;
};

int launch_fast(const Table &t, const FastPlanDev &pd, CandView c, double *d_val, double *d_dd,
                double *d_dk, cudaStream_t s, int tiers = 3, const TierEvents *ev = nullptr);
int heavy_grid_size(int device, unsigned *grid);
// Dynamic shared memory opt-in of the kernels holding the heavy tier's table (current device).
int heavy_smem_attributes();
int calibrate_issue(int device, double *thread_inst_per_s);
// Measured full-rate throughput of the three pipes the tier kernels use, in thread operations
// per second: FFMA (FMA pipe), MUFU sin/cos (XU pipe), DFMA (FP64 pipe).
int calibrate_pipes(int device, double *ffma_per_s, double *mufu_per_s, double *dfma_per_s);

}  // namespace mb
