/*
 * mertens_k2.h -- C-ABI of libmertens_k2.so, the B200 (sm_100a) evaluator of
 *
 *   K2(v, T, k) = 2 sum_{0<gamma<T} exp(-k gamma^2) Re( e^{i gamma v} / (rho zeta'(rho)) ),
 *   rho = 1/2 + i gamma,
 *
 * the zero sum of bzyzz/mertens_bound (README.md:28, THEOREM.md:7).
 *
 * Conventions
 *   - Plain pointers and sizes only.  Host-pointer entry points copy in and out on the
 *     table's own CUDA stream and return after the results are on the host.  *_dev entry
 *     points take device pointers and a cudaStream_t passed as void* and return without
 *     synchronising.
 *   - Every entry point returns an int status: MB_OK (0) or a negative MB_ERR_* code;
 *     mb_last_error() gives a message for the calling thread.  No entry point exits the
 *     process.  (The reference's evaluator has no error channel at all:
 *     search/path1_eval_fast.cpp:15,58 return void and check nothing.)
 *   - G_j = gamma_j / 2pi is unsigned 64.128 fixed point, passed as three u64 limbs per zero
 *     in the order [integer, fraction hi, fraction lo] (row-major n x 3).  The integer part
 *     must be < 2^32.
 *   - A candidate point is v = v_int + v_frac 2^-64 (+ an optional FP64 offset delta).
 *   - The cutoff T keeps the zeros with gamma_j < T (the table is sorted, so these are the
 *     first count_below(T) zeros); T = +inf keeps them all.
 *   - Outputs: val = K2, dd = dK2/ddelta (= dK2/dv), dk = dK2/dk.
 *   - A table handle must not be used by two host threads at the same time.
 */
#ifndef MERTENS_K2_H
#define MERTENS_K2_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MB_OK 0
#define MB_ERR_ARG (-1)      /* bad argument: null pointer, size or value out of range      */
#define MB_ERR_TABLE (-2)    /* table data rejected: unsorted gamma, non-finite c, G/gamma   */
#define MB_ERR_CUDA (-3)     /* CUDA runtime error                                          */
#define MB_ERR_TIMEOUT (-4)  /* a bounded device-side wait gave up                          */
#define MB_ERR_STATE (-5)    /* call made in the wrong state (e.g. plan for another table)  */
#define MB_ERR_CAPACITY (-6) /* request larger than a fixed capacity                        */

typedef struct mb_table mb_table;

/* Message for the last failed call on this thread ("" if none). */
const char *mb_last_error(void);

/* ABI version of this library (bumped on any signature change). */
int mb_abi_version(void);

/* Upload a zero table to device `device` and validate it.
 * Replaces the table loading of search/eval_tech1_600k.py:38-50 (load_zeros_bin) and
 * search/gpu_mertens_stream.cu:298-379 (ZeroData::load) -- those read a file; this takes the
 * arrays (the file formats are read by the Python host layer).
 * Rejected with MB_ERR_TABLE: gamma not strictly increasing or not finite/positive,
 * non-finite c, G integer part >= 2^32, or |gamma - 2pi G| > 4 ulp(gamma). */
int mb_table_create(const uint64_t *G3, const double *c_re, const double *c_im, const double *gamma,
                    int64_t n, int device, mb_table **out);
/* Fails with MB_ERR_STATE while plans created on the table are alive (destroy them first). */
int mb_table_destroy(mb_table *t);
int mb_table_size(const mb_table *t, int64_t *n_out);
/* Number of zeros with gamma < T. */
int mb_table_count_below(const mb_table *t, double T, int64_t *n_out);

/* Exact phase floor(frac(v G_j) 2^128) for every candidate and the first n_zeros zeros,
 * written row-major (P x n_zeros) as (hi, lo) words.  The hi word is floor(frac(v G) 2^64).
 * The reduction restated: search/path1_eval_fast.cpp:41-46 (128-bit fixed-point product,
 * top word kept) and legacy/superseded/certify_peak2_600k.py:183-187. */
int mb_phase128(mb_table *t, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                int64_t n_zeros, uint64_t *out_hi, uint64_t *out_lo);

/* Plain FP64 evaluation of K2 and its gradient: exact integer phase reduction, FP64
 * sine/cosine, FP64 accumulation.
 * Replaces search/path1_eval_fast.cpp:15-53 followed by the h0 sum at :76-81 (compute_peak_AB
 * then sum w A), and the term loop of certification/certify_K2.py:116-121 (point value). */
int mb_k2_plain(mb_table *t, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                const double *delta, double k, double T, double *out_val, double *out_dd,
                double *out_dk);
int mb_k2_plain_dev(mb_table *t, int64_t P, const uint64_t *d_v_int, const uint64_t *d_v_frac,
                    const double *d_delta, double k, double T, double *d_val, double *d_dd,
                    double *d_dk, void *stream);

/* Certified interval: out_lo[p] <= K2 <= out_hi[p] rigorously (directed rounding, Taylor
 * enclosures of sine/cosine with Lagrange remainders, CUDA exp() within 2 ulp) for the
 * table's exact G and c, v = v_int + v_frac 2^-64 widened by v_rad[p] (nullable) and each
 * term widened by 2 w term_rad[j] (nullable; n = count_below(T) entries, e.g. the radius of
 * c e^{i gamma v} implied by the input balls).  out_abs_hi (nullable) bounds sum 2 w |c|.
 * P <= 65535.  Replaces the ball sum of certification/certify_K2.py:100-133 (work) over all
 * batches and its serial reduction :179-192. */
int mb_k2_certified(mb_table *t, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                    const double *v_rad, double k, double T, const double *term_rad, double *out_lo,
                    double *out_hi, double *out_abs_hi);

/* Certified interval over the zeros [j0, j1) only, for k anywhere in [k_lo, k_hi] (a decimal
 * k such as 1.5e-10 is enclosed by its two neighbouring doubles).  term_rad (nullable) has
 * j1 - j0 entries.  The batch sum of certify_K2.work (certification/certify_K2.py:100-133) for
 * zeros n0 .. n0 + num - 1 is j0 = n0 - 1, j1 = n0 - 1 + num. */
int mb_k2_certified_range(mb_table *t, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                          const double *v_rad, double k_lo, double k_hi, int64_t j0, int64_t j1,
                          const double *term_rad, double *out_lo, double *out_hi, double *out_abs_hi);

/* Certified intervals of K2 and of both derivatives over the zeros [j0, j1), k anywhere in
 * [k_lo, k_hi]: out_lo / out_hi hold 3P entries, rows K2, dK2/ddelta (= dK2/dv =
 * -2 sum w gamma Im(c e^{i gamma v})) and dK2/dk (= -2 sum w gamma^2 Re(c e^{i gamma v})), each
 * enclosed rigorously from the same directed-rounding sine/cosine, weight and gamma intervals as
 * mb_k2_certified_range; v_rad and term_rad widen the derivative terms by the extra factors
 * gamma_hi and gamma_hi^2.  The derivatives of certification/certify_K2.py:116-121's term (that
 * script encloses only the value): the interval check of the gradients the chosen form returns. */
int mb_k2_certified_grad_range(mb_table *t, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                               const double *v_rad, double k_lo, double k_hi, int64_t j0, int64_t j1,
                               const double *term_rad, double *out_lo, double *out_hi);

/* Plain FP64 K2 for callers that cannot allocate device memory: no counterpart in the
 * reference (its evaluator is host code).  Callers in a host callback, inside a fixed memory
 * budget or in a runtime that owns every allocation cannot call cudaMalloc; this entry point
 * allocates nothing.  The caller passes the zero data as device arrays in the library's
 * layout -- d_g = five planar u32 limb arrays of G 2^128 (least significant first, stride
 * n_zeros), d_gamma, d_cre, d_cim -- sums the first n_use zeros, and passes candidates and
 * outputs as device arrays.  Scratch for the partial sums is a fixed 8 MiB device array that
 * every GPU loading the library keeps until exit, so P <= 349,525 (larger P returns
 * MB_ERR_CAPACITY).  All calls share that array: calls that overlap on the GPU (other streams,
 * other host threads) race on it.  The first call on a device (and the first after that
 * device's context was replaced, e.g. by cudaDeviceReset) looks up the array's address and sets
 * the plain kernel's shared-memory carveout; make it before any stream capture.  Runs on the
 * current device, asynchronously on `stream`. */
int mb_k2_plain_noalloc_dev(const uint32_t *d_g, const double *d_gamma, const double *d_cre,
                            const double *d_cim, int64_t n_zeros, int64_t n_use, int64_t P,
                            const uint64_t *d_v_int, const uint64_t *d_v_frac, const double *d_delta,
                            double k, double *d_val, double *d_dd, double *d_dk, void *stream);

/* ---- chosen form: batched, precision-tiered value + gradient ----------------------------
 * A plan fixes n_groups groups; group g is the next counts[g] candidates of the candidate
 * array, evaluated at (ks[g], Ts[g]).  Per group the zeros below T are split at a boundary
 * n_heavy chosen so that the a-priori worst-case error bound stays <= tol: the first n_heavy
 * zeros (the heavy tier) are summed in FP64 (64-bit phase, table sine/cosine with FP64
 * polynomials), the rest (the light tier) with a 32-bit phase, MUFU sine/cosine and FP32
 * accumulators that are added into FP64 partial sums every 32 terms.  Each tier is one kernel
 * over the work items of every group: the heavy kernel is persistent (two CTAs per SM pull items
 * from a counter) and runs on a second stream concurrently with the light kernel (one CTA per
 * item); a deterministic reduction adds the partial sums.  mb_plan_run replays a captured CUDA
 * graph of the whole sequence.
 * Replaces the candidate scoring loops of search/eval_tech1_600k.py:201-273,
 * search/eval_tech2_hdrop_600k.py:127-201 and search/eval_sub35_candidates.py:64-138 (which
 * call compute_peak_AB + polish_peaks_with_weights per weight vector), and the k-scan of
 * search/path1_kernel_opt.py:526,687. */
typedef struct mb_plan mb_plan;

int mb_plan_create(mb_table *t, int n_groups, const int64_t *counts, const double *ks,
                   const double *Ts, double tol, mb_plan **out);
/* Register a per-zero weight vector w[n] (n = table size) with the table; *slot names it.
 * The search drivers score the same candidates under several weights besides the Gaussians:
 * the Jurkat-Peyerimhoff kernel, raw (w = 1) and a first-10k cutoff
 * (search/eval_tech1_600k.py:243-249). */
int mb_table_add_weights(mb_table *t, const double *w, int64_t n, int *slot);
/* As mb_plan_create, with weight_slots[g] = a registered weight vector for group g, or -1 for
 * exp(-k_g gamma^2).  For a weight vector, dk returns -2 sum gamma^2 w Re(c e^{i gamma v}) =
 * d2K/ddelta2 (the Newton denominator); k_g is ignored. */
int mb_plan_create_weighted(mb_table *t, int n_groups, const int64_t *counts, const double *ks, const double *Ts,
                            const int *weight_slots, double tol, mb_plan **out);
int mb_plan_destroy(mb_plan *p);
/* Tail skip: give the share skip_frac (0 .. 0.25) of tol to not evaluating, per group, the zeros
 * beyond the point where the remaining sum of 2|c| w is <= skip_frac * tol (the Gaussian makes
 * most zeros below a large T negligible at tol = 1e-10: ~76% of them at T = 3e5, k = 3e-9).
 * The light tier fits in what remains of tol; the group bound includes the skipped sum; the
 * derivative outputs omit the same zeros.  0 (the default) evaluates every zero below T, as the
 * reference does.  No reference counterpart (it sums every zero below its cutoff). */
int mb_plan_set_skip(mb_plan *p, double skip_frac);
/* Autotuner: times every tile configuration (light_cpt in {2, 3, 4} x nzw_shift in {0, 1} x
 * chunk_scale in {0.5, 1, 2}, in that nesting order; timings, nullable, receives the 18 median
 * times in ms) with mb_plan_time(reps) under the plan's current schedule and applies the fastest.
 * The Python layer runs it under each schedule (mb_plan_set_schedule), keeps the fastest pair and
 * caches the choice per GPU and workload class.  No reference counterpart (its evaluator has no
 * tunables). */
int mb_plan_autotune(mb_plan *p, int reps, int *light_cpt, int *nzw_shift, double *chunk_scale, double *best_ms,
                     double *timings);
/* A-priori bounds of the absolute error of group g's outputs: K2 (the bound of
 * mb_plan_group_info), dK2/ddelta and dK2/dk (the same per-term errors applied to the amplitude
 * sums 2|c| w gamma and 2|c| w gamma^2, plus the skipped zeros' sums under a tail skip). */
int mb_plan_group_bounds(const mb_plan *p, int g, double *val, double *dd, double *dk);
/* Zeros evaluated for group g (count_below(T) without a tail skip). */
int mb_plan_group_zeros(const mb_plan *p, int g, int64_t *n_eval);
/* Override the tile shape of group g: cpt in {1,2,4} candidates per thread, nzw in {1,2,4,8}
 * warps splitting the zeros, chunk sizes in zeros (0 = automatic; multiples of 128 / 256). */
int mb_plan_set_shape(mb_plan *p, int g, int cpt, int nzw, int64_t heavy_chunk, int64_t light_chunk);
/* Plan-wide tile configuration, the autotuner's search space: light-kernel candidates per
 * thread (2, 3, 4), extra doublings of each group's warp split (0..3), and a scale of the
 * automatic work-item size (0.125..8).  Replaces per-group overrides. */
int mb_plan_configure(mb_plan *p, int light_cpt, int nzw_shift, double chunk_scale);
/* How the two tiers run: 0 (the default) launches the persistent heavy kernel on a second stream
 * concurrently with the light kernel (one CTA per item); 1 runs every item of both tiers in one
 * persistent kernel (two CTAs per SM pulling heavy items first, then light items, from one
 * counter); 2 is the same kernel with the items of both tiers in one list ordered by estimated
 * cost, largest first (a heavy term weighted 2.5 light terms), so the last items to start are the
 * smallest of either tier; 3 is the same kernel with one queue per tier: the first CTA on each SM
 * pulls heavy items, the second light items, and a CTA whose queue is empty takes the other's.
 * One-tier runs (mb_plan_run_tiers_dev 1 or 2) use the tier kernels in every schedule.  The
 * results are the same bits in every schedule.  The autotuner tries all four.  No reference
 * counterpart. */
int mb_plan_set_schedule(mb_plan *p, int schedule);
int mb_plan_schedule(const mb_plan *p, int *schedule);
/* Restrict every group to the zeros [j0, j1) of its [0, count_below(T)): one shard of a
 * zero-range split across GPUs; the shards' results add up to the whole sum (tier boundaries and
 * error bounds are those of the whole sum).  No reference counterpart (the reference shards zero
 * batches over a process pool, certification/certify_K2.py:160-174). */
int mb_plan_set_zero_range(mb_plan *p, int64_t j0, int64_t j1);
/* Median device time in ms of `reps` runs on synthetic candidates (for the autotuner). */
int mb_plan_time(mb_plan *p, int reps, double *ms);
int mb_plan_info(const mb_plan *p, int64_t *P, double *zero_terms, int *n_items);
/* *fused = 1 when the plan's light tier takes the fraction part of v through one FMA (every zero
 * of its table below gamma = 2 pi (2^19 - 1) = 3.29e6), 0 for the split form.  Plan introspection;
 * no counterpart in the reference. */
int mb_plan_light_form(const mb_plan *p, int *fused);
int mb_plan_group_info(const mb_plan *p, int g, int64_t *n_T, int64_t *n_heavy, double *err_bound,
                       double *sum_abs);
/* Device pointers (P = sum of counts), asynchronous on `stream`. */
int mb_plan_run_dev(mb_plan *p, const uint64_t *d_v_int, const uint64_t *d_v_frac,
                    const double *d_delta, double *d_val, double *d_dd, double *d_dk, void *stream);
/* Host pointers: copies through pinned staging and replays the plan's CUDA graph
 * (H2D, kernels, D2H); returns when the results are in val/dd/dk. */
int mb_plan_run(mb_plan *p, const uint64_t *v_int, const uint64_t *v_frac, const double *delta,
                double *val, double *dd, double *dk);
/* Run one tier only (tiers: 1 heavy, 2 light, 3 both = mb_plan_run_dev), to time a kernel on
 * its own; with 1 or 2 the results hold that tier's terms only (the other tier's partial sums are
 * cleared first).  No reference counterpart. */
int mb_plan_run_tiers_dev(mb_plan *p, int tiers, const uint64_t *d_v_int, const uint64_t *d_v_frac,
                          const double *d_delta, double *d_val, double *d_dd, double *d_dk, void *stream);
/* Zero-terms per run in each tier. */
int mb_plan_tier_terms(const mb_plan *p, double *heavy_terms, double *light_terms);
/* Measured full-rate instruction issue throughput of `device` (FFMA chains), in thread
 * instructions per second: the peak against which the ALU-bound kernels are reported. */
int mb_calibrate_issue(int device, double *thread_inst_per_s);
/* Measured full-rate throughput of `device`'s FMA pipe (FFMA), XU pipe (MUFU sin/cos) and FP64
 * pipe (DFMA), in thread operations per second (each output nullable): the pipe peaks against
 * which the tier kernels' algorithmic work is reported.  No reference counterpart. */
int mb_calibrate_pipes(int device, double *ffma_per_s, double *mufu_per_s, double *dfma_per_s);
/* Per-kernel timing hook: with n_slots > 0, every later mb_plan_run_dev / mb_plan_run_tiers_dev
 * records CUDA events around its light-tier launch (on the caller's stream) and its heavy-tier
 * launch (on the stream it runs on) into a ring of n_slots slots; 0 turns it off.  The plan's
 * host-pointer runs (its CUDA graph) record nothing.  No reference counterpart. */
int mb_plan_kernel_timing(mb_plan *p, int n_slots);
/* The light and heavy kernel times (ms) of the last min(n, n_slots, runs) timed runs, oldest
 * first, in light_ms / heavy_ms (-1 where that tier did not run); *n_out = how many.  Under a
 * one-kernel schedule (mb_plan_set_schedule 1, 2 or 3) a run of both tiers is one launch: its time
 * is in light_ms and heavy_ms is -1.  Waits for those runs' events. */
int mb_plan_kernel_times(mb_plan *p, int n, double *light_ms, double *heavy_ms, int *n_out);

/* Batched Newton polish of the offsets: h0 = K2 at the given d_delta; then up to `iters` steps
 * delta -= clamp(K2'/K2'', +-max_step) with K2' = dK2/ddelta, K2'' = d2K2/ddelta2 = dK2/dk from
 * the fused kernel; a candidate stops after |step| < 1e-13 or |K2''| <= 1e-12; the larger |K2|
 * of start and end point is kept.  d_delta is updated in place; d_val/d_dd/d_dk hold the kept
 * point's values.  Restates the Newton loop of search/path1_eval_fast.cpp:103-141 (there:
 * 6 steps, clamp 1e-4) on the chosen form. */
int mb_plan_newton_dev(mb_plan *p, const uint64_t *d_v_int, const uint64_t *d_v_frac, double *d_delta,
                       int iters, double max_step, double *d_h0, double *d_val, double *d_dd, double *d_dk,
                       void *stream);

/* One-group convenience: plan, run, destroy.  *err_bound receives the a-priori bound. */
int mb_k2_fast(mb_table *t, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
               const double *delta, double k, double T, double tol, double *out_val, double *out_dd,
               double *out_dk, double *err_bound);

/* Grid scan: out_h[p * n_m + i] = K2(v_p + (m0 + i) step) for i < n_m, with step the 64.64
 * fixed-point number step_int + step_frac 2^-64.  Every grid point's phase is exact
 * (frac(y G) = frac(v G) + m frac(step G), 128-bit); sine/cosine and sums in FP64.
 * Replaces the FP64 grid of search/polish.py:50-72 (phi + m dphi mod 2pi) and the grid stages
 * of search/gpu_mertens_stream.cu:381-505 / path1_eval_fast.cpp:86-101. */
int mb_grid_scan(mb_table *t, int64_t P, const uint64_t *v_int, const uint64_t *v_frac, double k, double T,
                 uint64_t step_int, uint64_t step_frac, int64_t m0, int64_t n_m, double *out_h);

/* Many small grids: out_h[p * n_m + i] = K2 over the first n_use zeros at v_p + (m0 + i) step,
 * n_m <= 1024, one CTA per base point.  The stage scans of the enumerators' hit polish
 * (search/gpu_mertens_stream.cu:381-505 ZeroData::polish, search/fast_mertens_enum.cpp:145-276:
 * 256, 512, 2048, 15000 and all zeros at decreasing steps) are calls of this. */
int mb_hit_scan(mb_table *t, int64_t P, const uint64_t *v_int, const uint64_t *v_frac, double k, int64_t n_use,
                uint64_t step_int, uint64_t step_frac, int64_t m0, int64_t n_m, double *out_h);

/* Staged leaf screen of the lattice enumerators: for each leaf v_p (64.64) and m = -3..3,
 * S_m = sum_j 2|c_j| e^{-k gamma_j^2} cos(2 pi frac((v_p + m step) G_j) + arg c_j) over the first
 * stage_end[s] zeros; a leaf passes stage s if max_m |S_m| >= threshold[s] and is a hit if it
 * passes every stage (stage_end increasing, at most 1024 zeros, at most 8 stages).  Hits are
 * returned in ascending leaf order in out_hits[*n_hits] with their per-stage scores
 * (out_hit_scores, n_stages per hit); out_scores (nullable, P x n_stages) receives every leaf's
 * scores, -1 for stages not reached.  More than max_hits hits: MB_ERR_CAPACITY with *n_hits =
 * the total (the kept subset is then arbitrary).  Replaces ZeroData::fast_screen
 * (search/fast_mertens_enum.cpp:108-142: 64/128 zeros, thresholds 0.810/0.875) and the GPU leaf
 * scoring (search/gpu_mertens_stream.cu:192-250: 64/128/256 zeros, 0.78/0.855/0.892), which take
 * cos from an FP32 table at a 12/14-bit phase; here the 32-bit phase and exact offsets make the
 * scores accurate to ~1e-6 of sum|a|. */
int mb_screen(mb_table *t, int64_t P, const uint64_t *v_int, const uint64_t *v_frac, double k, uint64_t step_int,
              uint64_t step_frac, int n_stages, const int64_t *stage_end, const float *threshold, int64_t max_hits,
              int64_t *out_hits, float *out_hit_scores, int64_t *n_hits, float *out_scores);
/* mb_screen on device leaves, asynchronous on `stream` (the GPU enumerator's loop,
 * search/gpu_mertens_stream.cu:192-250, scores leaves it generated on the device): d_v_int and
 * d_v_frac hold P leaves; stage_end and threshold are host arrays as above.  Hits go to d_hits /
 * d_hit_scores (device, at most max_hits, in arbitrary order) and their total to *d_n_hits (device;
 * above max_hits the kept subset is arbitrary); d_scores (device, nullable, P x n_stages) as
 * out_scores.  The zero records are staged in a buffer of the table that only mb_screen_dev uses,
 * so other calls on the table (on its own stream) cannot disturb a screen in flight; two
 * mb_screen_dev calls on one table that overlap on the GPU (different streams) race on it. */
int mb_screen_dev(mb_table *t, int64_t P, const uint64_t *d_v_int, const uint64_t *d_v_frac, double k,
                  uint64_t step_int, uint64_t step_frac, int n_stages, const int64_t *stage_end,
                  const float *threshold, int64_t max_hits, int64_t *d_hits, float *d_hit_scores,
                  unsigned long long *d_n_hits, float *d_scores, void *stream);

/* ---- per-peak polish contracts of search/path1_kernel_opt.py ------------------------------
 * A_j, B_j = 2 Re, 2 Im of c_j e^{i gamma_j y} and h(ddy) = sum_j w_j (A_j cos(gamma_j ddy) -
 * B_j sin(gamma_j ddy)).  Matrices are row-major (n_peaks, n_zeros) host arrays. */

/* out_A/out_B (P x n_zeros) at y = v + delta from the exact 128-bit phase; angle error below
 * 2 pi (|delta| 2^-52 + 2^-100), so A, B carry only FP64 sincos and product rounding.
 * |delta| <= 2^16.  Replaces compute_exact_mpfr_AB (search/path1_kernel_opt.py:71-91: one y,
 * 256-bit mpfr phase, rounded to FP64). */
int mb_exact_AB(mb_table *t, int64_t P, const uint64_t *v_int, const uint64_t *v_frac, const double *delta,
                int64_t n_zeros, double *out_A, double *out_B);

/* polish_single_peak (search/path1_kernel_opt.py:94-147) for each of n_peaks rows (row stride ld,
 * first n_zeros columns used): h0 = sum w A; grid ddy = numpy.linspace(-grid_hw, grid_hw,
 * 2 grid_steps + 1) over all n_zeros (none if grid_steps = 0), first argmax of |h|; Newton
 * (8 steps, clamp 2e-5, stop below 1e-14 or |h''| <= 1e-12) from 0 and from the grid's best;
 * a start's h is kept only if |h| > the best so far (which starts at h0, ddy 0). */
int mb_polish_single_peak(int64_t n_peaks, int64_t n_zeros, int64_t ld, const double *A, const double *B,
                          const double *gamma, const double *w, double grid_hw, int grid_steps,
                          double *out_h_unpol, double *out_h_pol, double *out_ddy_pol);

/* fast_polish_batch_blas (search/path1_kernel_opt.py:150-221): degree-16 Taylor moments of h in
 * u = gamma 1e-4 around ddy = 0 evaluated on ddy_grid (first argmax of |h|), h_unpol = the
 * zeroth moment; then exact Newton (4 steps, clamp 1e-5, stop below 1e-13) from the grid point
 * on the `top` peaks of largest |h_pol| (the reference uses 25; equal |h| in index order): a
 * peak keeps (h, ddy) if |h| > |h_unpol|, else (h_unpol, 0). */
int mb_fast_polish_batch(int64_t n_peaks, int64_t n_zeros, const double *A, const double *B, const double *gamma,
                         const double *w, const double *ddy_grid, int64_t n_grid, int top, double *out_h_unpol,
                         double *out_h_pol, double *out_ddy_pol);

/* The two polishes with (A_j, B_j) of peak p computed on the fly at y = v_p + delta_p as in
 * mb_exact_AB (no P x N matrices), over the table's first n_zeros zeros, gamma = the table's
 * FP64 gamma and w = a weight vector registered by mb_table_add_weights. */
int mb_polish_single_exact(mb_table *t, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                           const double *delta, int64_t n_zeros, int weight_slot, double grid_hw, int grid_steps,
                           double *out_h_unpol, double *out_h_pol, double *out_ddy_pol);
/* polish_peaks_with_weights (search/path1_eval_fast.cpp:58-143: h0; grid of 2 grid_steps + 1
 * shifts over the first min(n, 4096) zeros; <= 6 Newton steps, clamp 1e-4) for every candidate,
 * with (A_j, B_j) computed on the fly as in mb_exact_AB instead of read from P x N matrices:
 * the search drivers' compute_peak_AB + polish per weight vector (search/eval_tech1_600k.py:216-273)
 * without the matrices. */
int mb_polish_peaks_exact(mb_table *t, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                          const double *delta, int64_t n_zeros, int weight_slot, double grid_half_width,
                          int grid_steps, double *out_h_unpol, double *out_h_pol, double *out_ddy_pol);
/* mb_polish_peaks_exact under n_weights registered weight vectors at once (outputs n_weights x P,
 * row w for weight_slots[w]; each row equals the single-weight call).  The search drivers' step
 * (search/eval_tech1_600k.py:216-273: compute_peak_AB once, then polish_peaks_with_weights per
 * weight vector): the exact (A, B) of up to 65,535 peaks at a time is written once to a device
 * buffer of at most 4 GiB and at most half of the device's free memory, allocated for the call and
 * freed before it returns, and read by every weight's polish. */
int mb_polish_peaks_weights(mb_table *t, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                            const double *delta, int64_t n_zeros, int n_weights, const int *weight_slots,
                            double grid_half_width, int grid_steps, double *out_h_unpol, double *out_h_pol,
                            double *out_ddy_pol);
int mb_fast_polish_exact(mb_table *t, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                         const double *delta, int64_t n_zeros, int weight_slot, const double *ddy_grid,
                         int64_t n_grid, int top, double *out_h_unpol, double *out_h_pol, double *out_ddy_pol);

/* ---- compatibility with the reference's libpath1_eval.so ---------------------------------
 * Same names, signatures and host-array contracts as search/path1_eval_fast.cpp:15 and :58, so
 * search/eval_tech1_600k.py, eval_tech2_hdrop_600k.py, eval_sub35_candidates.py and
 * path1_kernel_opt.py can load this library instead.  Computed on the current CUDA device.
 * The void forms (like the reference) cannot return a status: on failure they print the
 * message to stderr and fill their outputs with NaN.  The mb_ forms return the status. */
void compute_peak_AB(int n_peaks, const uint64_t *x_lo_arr, const uint64_t *x_hi_arr, const double *dy0_arr,
                     int n_zeros, const double *alpha, const double *gamma, const uint64_t *ghi_lo,
                     const uint64_t *ghi_hi, const uint64_t *glo_lo, const uint64_t *glo_hi,
                     const uint64_t *psi_lo, const uint64_t *psi_hi, double *out_A, double *out_B);
void polish_peaks_with_weights(int n_peaks, int n_zeros, const double *A, const double *B, const double *gamma,
                               const double *w, double grid_half_width, int grid_steps, double *out_h_unpol,
                               double *out_h_pol, double *out_ddy_pol);
int mb_compute_peak_AB(int n_peaks, const uint64_t *x_lo_arr, const uint64_t *x_hi_arr, const double *dy0_arr,
                       int n_zeros, const double *alpha, const double *gamma, const uint64_t *ghi_lo,
                       const uint64_t *ghi_hi, const uint64_t *glo_lo, const uint64_t *glo_hi,
                       const uint64_t *psi_lo, const uint64_t *psi_hi, double *out_A, double *out_B);
int mb_polish_peaks_with_weights(int n_peaks, int n_zeros, const double *A, const double *B, const double *gamma,
                                 const double *w, double grid_half_width, int grid_steps, double *out_h_unpol,
                                 double *out_h_pol, double *out_ddy_pol);

#ifdef __cplusplus
}
#endif
#endif /* MERTENS_K2_H */
