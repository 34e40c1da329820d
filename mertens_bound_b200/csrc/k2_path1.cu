// The per-peak polish contracts of search/path1_kernel_opt.py on the GPU:
//   compute_exact_mpfr_AB   (:71-91)   -> mb_exact_AB: A_j, B_j = 2 c_j e^{i gamma_j y} from the exact
//                                         128-bit phase (the reference rounds a 256-bit mpfr product)
//   polish_single_peak      (:94-147)  -> mb_polish_single_peak (A/B rows) and
//                                         mb_polish_single_exact (A/B computed on the fly)
//   fast_polish_batch_blas  (:150-221) -> mb_fast_polish_batch (A/B rows) and
//                                         mb_fast_polish_exact (A/B computed on the fly)
// and, for the search drivers' polish_peaks_with_weights (search/path1_eval_fast.cpp:58-143, whose
// A/B form is in k2_compat.cu), mb_polish_peaks_exact with (A, B) computed on the fly.
// The *_exact forms read the table and the peaks' 64.64 fixed-point v (+ delta) and never form the
// P x N matrices, so they are bound by the phase and sincos work, not by 16 B/term of HBM traffic.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "k2_polish.cuh"

namespace mb {
namespace {

// one cluster of POLISH_CLUSTER CTAs per peak: the grid stays within 2^31 - 1 CTAs
constexpr int64_t MAX_POLISH_PEAKS = (int64_t)1 << 26;

__global__ void exact_ab_kernel(ABExact src, int64_t n, int64_t p0, double *A, double *B) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int64_t p = p0 + blockIdx.y;
    const ABExact::Peak pk = src.peak(p);
    double a, b;
    src.at(pk, j, a, b);
    const size_t o = (size_t)blockIdx.y * n + j;
    A[o] = a;
    B[o] = b;
}

// numpy.linspace(-hw, hw, 2 steps + 1) value for value: arange(num) * step + start, last = stop.
std::vector<double> linspace_grid(double hw, int steps) {
    std::vector<double> g;
    if (steps <= 0) return g;
    const int num = 2 * steps + 1;
    const double start = -hw, step = (hw - start) / (double)(num - 1);
    g.resize(num);
    for (int i = 0; i < num; ++i) {
        volatile double t = (double)i * step;   // two roundings, as numpy does
        g[i] = t + start;
    }
    g[num - 1] = hw;
    return g;
}

// Indices of the `top` largest |h|, largest first; equal |h| in index order.
std::vector<int> top_indices(const double *h, int64_t P, int top) {
    std::vector<int> idx(P);
    std::iota(idx.begin(), idx.end(), 0);
    const int k = (int)std::min<int64_t>(top, P);
    std::partial_sort(idx.begin(), idx.begin() + k, idx.end(), [h](int a, int b) {
        const double x = std::fabs(h[a]), y = std::fabs(h[b]);
        return x > y || (x == y && a < b);
    });
    idx.resize(k);
    return idx;
}

int check_grid(const double *grid, int64_t n_grid, const char *who) {
    MB_CHECK_ARG(grid != nullptr && n_grid >= 1 && n_grid <= (1 << 20), "%s: n_grid=%lld", who, (long long)n_grid);
    for (int64_t i = 0; i < n_grid; ++i)
        MB_CHECK_ARG(std::isfinite(grid[i]), "%s: grid[%lld] is not finite", who, (long long)i);
    return MB_OK;
}

int check_peaks(const mb::Table &t, int64_t P, const uint64_t *vi, const uint64_t *vf, const double *delta,
                int64_t n_zeros, const char *who) {
    MB_CHECK_ARG(vi && vf, "%s: null candidate array", who);
    MB_CHECK_ARG(P >= 0 && P <= ((int64_t)1 << 30), "%s: P=%lld", who, (long long)P);
    MB_CHECK_ARG(n_zeros >= 0 && n_zeros <= t.n, "%s: n_zeros=%lld of %lld", who, (long long)n_zeros,
                 (long long)t.n);
    if (delta)
        for (int64_t p = 0; p < P; ++p)
            MB_CHECK_ARG(std::isfinite(delta[p]) && std::fabs(delta[p]) <= 65536.0,
                         "%s: delta[%lld]=%g must be finite with |delta| <= 2^16", who, (long long)p, delta[p]);
    return MB_OK;
}

int check_weights(const mb::Table &t, int slot, const char *who) {
    MB_CHECK_ARG(slot >= 0 && slot < (int)t.d_weights.size(), "%s: weight slot %d not registered", who, slot);
    return MB_OK;
}

// Candidates, grid, outputs and selection staged in the table's io buffer.
struct ExactStage {
    uint64_t *vi, *vf;
    double *delta, *grid, *hu, *hp, *dp;
    int *sel;
};

int stage_exact(Table &t, int64_t P, const uint64_t *vi, const uint64_t *vf, const double *delta,
                const double *grid, int64_t n_grid, int top, ExactStage &s) {
    const size_t need = 6 * ((size_t)P * 8 + 256) + ((size_t)n_grid * 8 + 256) + ((size_t)top * 4 + 256) + 256;
    MB_TRY(t.io.ensure(need));
    char *p = (char *)t.io.p;
    s.vi = carve<uint64_t>(p, P);
    s.vf = carve<uint64_t>(p, P);
    s.delta = carve<double>(p, P);
    s.hu = carve<double>(p, P);
    s.hp = carve<double>(p, P);
    s.dp = carve<double>(p, P);
    s.grid = carve<double>(p, n_grid);
    s.sel = carve<int>(p, top);
    MB_CUDA(cudaMemcpyAsync(s.vi, vi, P * 8, cudaMemcpyHostToDevice, t.stream));
    MB_CUDA(cudaMemcpyAsync(s.vf, vf, P * 8, cudaMemcpyHostToDevice, t.stream));
    if (delta)
        MB_CUDA(cudaMemcpyAsync(s.delta, delta, P * 8, cudaMemcpyHostToDevice, t.stream));
    else
        MB_CUDA(cudaMemsetAsync(s.delta, 0, P * 8, t.stream));
    if (n_grid > 0) MB_CUDA(cudaMemcpyAsync(s.grid, grid, n_grid * 8, cudaMemcpyHostToDevice, t.stream));
    return MB_OK;
}

int fetch_outputs(cudaStream_t st, int64_t P, const double *hu, const double *hp, const double *dp, double *out_hu,
                  double *out_hp, double *out_dp) {
    MB_CUDA(cudaMemcpyAsync(out_hu, hu, P * 8, cudaMemcpyDeviceToHost, st));
    MB_CUDA(cudaMemcpyAsync(out_hp, hp, P * 8, cudaMemcpyDeviceToHost, st));
    MB_CUDA(cudaMemcpyAsync(out_dp, dp, P * 8, cudaMemcpyDeviceToHost, st));
    MB_CUDA(cudaStreamSynchronize(st));
    return MB_OK;
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" int mb_exact_AB(mb_table *h, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                           const double *delta, int64_t n_zeros, double *out_A, double *out_B) {
    MB_CHECK_ARG(h && out_A && out_B, "mb_exact_AB: null argument");
    Table &t = table_of(h);
    MB_TRY(check_peaks(t, P, v_int, v_frac, delta, n_zeros, "mb_exact_AB"));
    if (P == 0 || n_zeros == 0) return MB_OK;
    MB_TRY(device_guard(t.device));
    const size_t N = (size_t)n_zeros;
    // peaks per pass: A/B slabs within 2 GiB, grid.y within 65535
    const int64_t chunk = (int64_t)std::max<size_t>(
        1, std::min<size_t>({(size_t)P, ((size_t)1 << 31) / (16 * N), (size_t)65535}));
    ExactStage s;
    MB_TRY(stage_exact(t, P, v_int, v_frac, delta, nullptr, 0, 0, s));
    MB_TRY(t.work.ensure(2 * ((size_t)chunk * N * 8 + 256)));
    char *wp = (char *)t.work.p;
    double *d_A = carve<double>(wp, chunk * N), *d_B = carve<double>(wp, chunk * N);
    const ABExact src{view(t), s.vi, s.vf, s.delta};
    for (int64_t p0 = 0; p0 < P; p0 += chunk) {
        const int64_t np = std::min(chunk, P - p0);
        dim3 grid((unsigned)((N + 255) / 256), (unsigned)np);
        exact_ab_kernel<<<grid, 256, 0, t.stream>>>(src, n_zeros, p0, d_A, d_B);
        MB_CUDA(cudaGetLastError());
        MB_CUDA(cudaMemcpyAsync(out_A + p0 * N, d_A, np * N * 8, cudaMemcpyDeviceToHost, t.stream));
        MB_CUDA(cudaMemcpyAsync(out_B + p0 * N, d_B, np * N * 8, cudaMemcpyDeviceToHost, t.stream));
    }
    MB_CUDA(cudaStreamSynchronize(t.stream));
    return MB_OK;
}

extern "C" int mb_polish_single_peak(int64_t n_peaks, int64_t n_zeros, int64_t ld, const double *A, const double *B,
                                     const double *gamma, const double *w, double grid_hw, int grid_steps,
                                     double *out_h_unpol, double *out_h_pol, double *out_ddy_pol) {
    const char *who = "mb_polish_single_peak";
    MB_CHECK_ARG(n_peaks >= 0 && n_zeros >= 0 && ld >= n_zeros && grid_steps >= 0 && grid_steps <= (1 << 19),
                 "%s: bad sizes", who);
    if (n_peaks == 0) return MB_OK;
    MB_CHECK_ARG(A && B && gamma && w && out_h_unpol && out_h_pol && out_ddy_pol, "%s: null array", who);
    MB_CHECK_ARG(std::isfinite(grid_hw), "%s: grid_hw is not finite", who);
    const std::vector<double> grid = linspace_grid(grid_hw, grid_steps);
    std::lock_guard<std::mutex> lock(scratch_mutex());
    const size_t N = (size_t)std::max<int64_t>(n_zeros, 1), G = std::max<size_t>(grid.size(), 1);
    const int64_t chunk = (int64_t)std::max<size_t>(1, std::min<size_t>((size_t)n_peaks, ((size_t)1 << 31) / (16 * N)));
    const size_t bytes = 2 * (N * 8 + 256) + (G * 8 + 256) + 2 * ((size_t)chunk * N * 8 + 256) +
                         3 * ((size_t)chunk * 8 + 256);
    void *base = nullptr;
    MB_TRY(scratch_buffer(bytes, &base));
    char *p = (char *)base;
    double *d_g = carve<double>(p, N), *d_w = carve<double>(p, N), *d_grid = carve<double>(p, G);
    double *d_A = carve<double>(p, chunk * N), *d_B = carve<double>(p, chunk * N);
    double *d_hu = carve<double>(p, chunk), *d_hp = carve<double>(p, chunk), *d_dp = carve<double>(p, chunk);
    cudaStream_t s = cudaStreamPerThread;
    if (n_zeros > 0) {
        MB_CUDA(cudaMemcpyAsync(d_g, gamma, n_zeros * 8, cudaMemcpyHostToDevice, s));
        MB_CUDA(cudaMemcpyAsync(d_w, w, n_zeros * 8, cudaMemcpyHostToDevice, s));
    }
    if (!grid.empty()) MB_CUDA(cudaMemcpyAsync(d_grid, grid.data(), grid.size() * 8, cudaMemcpyHostToDevice, s));
    for (int64_t p0 = 0; p0 < n_peaks; p0 += chunk) {
        const int64_t np = std::min(chunk, n_peaks - p0);
        if (n_zeros > 0) {
            MB_CUDA(cudaMemcpy2DAsync(d_A, n_zeros * 8, A + p0 * ld, ld * 8, n_zeros * 8, np, cudaMemcpyHostToDevice, s));
            MB_CUDA(cudaMemcpy2DAsync(d_B, n_zeros * 8, B + p0 * ld, ld * 8, n_zeros * 8, np, cudaMemcpyHostToDevice, s));
        }
        PolishArgs a{n_zeros, d_g, d_w, d_grid, (int)grid.size(), 0.0, nullptr, d_hu, d_hp, d_dp};
        peak_polish_kernel<ABMatrix, POLISH_SINGLE><<<(unsigned)(np * POLISH_CLUSTER), POLISH_THREADS, 0, s>>>(ABMatrix{d_A, d_B, n_zeros}, a);
        MB_CUDA(cudaGetLastError());
        MB_CUDA(cudaMemcpyAsync(out_h_unpol + p0, d_hu, np * 8, cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaMemcpyAsync(out_h_pol + p0, d_hp, np * 8, cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaMemcpyAsync(out_ddy_pol + p0, d_dp, np * 8, cudaMemcpyDeviceToHost, s));
    }
    MB_CUDA(cudaStreamSynchronize(s));
    return MB_OK;
}

extern "C" int mb_fast_polish_batch(int64_t n_peaks, int64_t n_zeros, const double *A, const double *B,
                                    const double *gamma, const double *w, const double *ddy_grid, int64_t n_grid,
                                    int top, double *out_h_unpol, double *out_h_pol, double *out_ddy_pol) {
    const char *who = "mb_fast_polish_batch";
    MB_CHECK_ARG(n_peaks >= 0 && n_zeros >= 0 && top >= 0 && top <= 65536, "%s: bad sizes", who);
    if (n_peaks == 0) return MB_OK;
    MB_CHECK_ARG(A && B && gamma && w && out_h_unpol && out_h_pol && out_ddy_pol, "%s: null array", who);
    MB_TRY(check_grid(ddy_grid, n_grid, who));
    std::lock_guard<std::mutex> lock(scratch_mutex());
    const size_t N = (size_t)std::max<int64_t>(n_zeros, 1);
    const int64_t chunk = (int64_t)std::max<size_t>(1, std::min<size_t>((size_t)n_peaks, ((size_t)1 << 31) / (16 * N)));
    const int64_t nsel = std::min<int64_t>(top, n_peaks);
    const size_t bytes = 2 * (N * 8 + 256) + ((size_t)n_grid * 8 + 256) + 2 * ((size_t)chunk * N * 8 + 256) +
                         3 * ((size_t)n_peaks * 8 + 256);
    void *base = nullptr;
    MB_TRY(scratch_buffer(bytes, &base));
    char *p = (char *)base;
    double *d_g = carve<double>(p, N), *d_w = carve<double>(p, N), *d_grid = carve<double>(p, n_grid);
    double *d_A = carve<double>(p, chunk * N), *d_B = carve<double>(p, chunk * N);
    double *d_hu = carve<double>(p, n_peaks), *d_hp = carve<double>(p, n_peaks), *d_dp = carve<double>(p, n_peaks);
    cudaStream_t s = cudaStreamPerThread;
    if (n_zeros > 0) {
        MB_CUDA(cudaMemcpyAsync(d_g, gamma, n_zeros * 8, cudaMemcpyHostToDevice, s));
        MB_CUDA(cudaMemcpyAsync(d_w, w, n_zeros * 8, cudaMemcpyHostToDevice, s));
    }
    MB_CUDA(cudaMemcpyAsync(d_grid, ddy_grid, n_grid * 8, cudaMemcpyHostToDevice, s));
    for (int64_t p0 = 0; p0 < n_peaks; p0 += chunk) {
        const int64_t np = std::min(chunk, n_peaks - p0);
        if (n_zeros > 0) {
            MB_CUDA(cudaMemcpyAsync(d_A, A + p0 * N, np * N * 8, cudaMemcpyHostToDevice, s));
            MB_CUDA(cudaMemcpyAsync(d_B, B + p0 * N, np * N * 8, cudaMemcpyHostToDevice, s));
        }
        MomentArgs m{n_zeros, d_g, d_w, d_grid, (int)n_grid, d_hu + p0, d_hp + p0, d_dp + p0};
        taylor_moments_kernel<ABMatrix><<<(unsigned)(np * POLISH_CLUSTER), POLISH_THREADS, 0, s>>>(ABMatrix{d_A, d_B, n_zeros}, m);
        MB_CUDA(cudaGetLastError());
    }
    MB_TRY(fetch_outputs(s, n_peaks, d_hu, d_hp, d_dp, out_h_unpol, out_h_pol, out_ddy_pol));
    if (nsel == 0) return MB_OK;
    // exact Newton on the top peaks: their rows gathered into the first slab rows
    const std::vector<int> sel = top_indices(out_h_pol, n_peaks, (int)nsel);
    for (int64_t done = 0; done < nsel; done += chunk) {
        const int64_t np = std::min(chunk, nsel - done);
        for (int64_t r = 0; r < np; ++r) {
            const int64_t q = sel[done + r];
            if (n_zeros > 0) {
                MB_CUDA(cudaMemcpyAsync(d_A + r * N, A + q * N, N * 8, cudaMemcpyHostToDevice, s));
                MB_CUDA(cudaMemcpyAsync(d_B + r * N, B + q * N, N * 8, cudaMemcpyHostToDevice, s));
            }
            MB_CUDA(cudaMemcpyAsync(d_hu + r, out_h_unpol + q, 8, cudaMemcpyHostToDevice, s));
            MB_CUDA(cudaMemcpyAsync(d_dp + r, out_ddy_pol + q, 8, cudaMemcpyHostToDevice, s));
        }
        PolishArgs a{n_zeros, d_g, d_w, nullptr, 0, 0.0, nullptr, d_hu, d_hp, d_dp};
        peak_polish_kernel<ABMatrix, POLISH_TOPK><<<(unsigned)(np * POLISH_CLUSTER), POLISH_THREADS, 0, s>>>(ABMatrix{d_A, d_B, n_zeros}, a);
        MB_CUDA(cudaGetLastError());
        std::vector<double> hp(np), dp(np);
        MB_CUDA(cudaMemcpyAsync(hp.data(), d_hp, np * 8, cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaMemcpyAsync(dp.data(), d_dp, np * 8, cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaStreamSynchronize(s));
        for (int64_t r = 0; r < np; ++r) {
            out_h_pol[sel[done + r]] = hp[r];
            out_ddy_pol[sel[done + r]] = dp[r];
        }
    }
    return MB_OK;
}

extern "C" int mb_polish_single_exact(mb_table *h, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                                      const double *delta, int64_t n_zeros, int weight_slot, double grid_hw,
                                      int grid_steps, double *out_h_unpol, double *out_h_pol, double *out_ddy_pol) {
    const char *who = "mb_polish_single_exact";
    MB_CHECK_ARG(h && out_h_unpol && out_h_pol && out_ddy_pol, "%s: null argument", who);
    MB_CHECK_ARG(P <= MAX_POLISH_PEAKS, "%s: P=%lld above %lld peaks per call", who, (long long)P,
                 (long long)MAX_POLISH_PEAKS);
    Table &t = table_of(h);
    MB_TRY(check_peaks(t, P, v_int, v_frac, delta, n_zeros, who));
    MB_TRY(check_weights(t, weight_slot, who));
    MB_CHECK_ARG(grid_steps >= 0 && grid_steps <= (1 << 19) && std::isfinite(grid_hw), "%s: bad grid", who);
    if (P == 0) return MB_OK;
    MB_TRY(device_guard(t.device));
    const std::vector<double> grid = linspace_grid(grid_hw, grid_steps);
    ExactStage s;
    MB_TRY(stage_exact(t, P, v_int, v_frac, delta, grid.data(), (int64_t)grid.size(), 0, s));
    PolishArgs a{n_zeros, t.d_gamma, t.d_weights[weight_slot], s.grid, (int)grid.size(), 0.0, nullptr, s.hu, s.hp, s.dp};
    peak_polish_kernel<ABExact, POLISH_SINGLE><<<(unsigned)(P * POLISH_CLUSTER), POLISH_THREADS, 0, t.stream>>>(
        ABExact{view(t), s.vi, s.vf, s.delta}, a);
    MB_CUDA(cudaGetLastError());
    return fetch_outputs(t.stream, P, s.hu, s.hp, s.dp, out_h_unpol, out_h_pol, out_ddy_pol);
}

extern "C" int mb_polish_peaks_exact(mb_table *h, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                                     const double *delta, int64_t n_zeros, int weight_slot, double grid_half_width,
                                     int grid_steps, double *out_h_unpol, double *out_h_pol, double *out_ddy_pol) {
    const char *who = "mb_polish_peaks_exact";
    MB_CHECK_ARG(h && out_h_unpol && out_h_pol && out_ddy_pol, "%s: null argument", who);
    MB_CHECK_ARG(P <= MAX_POLISH_PEAKS, "%s: P=%lld above %lld peaks per call", who, (long long)P,
                 (long long)MAX_POLISH_PEAKS);
    Table &t = table_of(h);
    MB_TRY(check_peaks(t, P, v_int, v_frac, delta, n_zeros, who));
    MB_TRY(check_weights(t, weight_slot, who));
    MB_CHECK_ARG(grid_steps >= 0 && grid_steps <= (1 << 19) && std::isfinite(grid_half_width), "%s: bad grid", who);
    if (P == 0) return MB_OK;
    MB_TRY(device_guard(t.device));
    ExactStage s;
    MB_TRY(stage_exact(t, P, v_int, v_frac, delta, nullptr, 0, 0, s));
    PolishArgs a{n_zeros, t.d_gamma, t.d_weights[weight_slot], nullptr, grid_steps, grid_half_width, nullptr,
                 s.hu, s.hp, s.dp};
    peak_polish_kernel<ABExact, POLISH_EVAL_FAST><<<(unsigned)(P * POLISH_CLUSTER), POLISH_THREADS, 0, t.stream>>>(
        ABExact{view(t), s.vi, s.vf, s.delta}, a);
    MB_CUDA(cudaGetLastError());
    return fetch_outputs(t.stream, P, s.hu, s.hp, s.dp, out_h_unpol, out_h_pol, out_ddy_pol);
}

// polish_peaks_with_weights under several weight vectors: the exact (A, B) of a chunk of peaks is
// written once to HBM (the reference's P x N matrices, search/eval_tech1_600k.py:216-273, with the
// exact phase of mb_exact_AB) and every weight's polish reads it, instead of recomputing each term's
// 128-bit phase and sine/cosine in every pass.  Chunks keep the matrices within AB_BUDGET bytes.
constexpr size_t AB_BUDGET = (size_t)4 << 30;

extern "C" int mb_polish_peaks_weights(mb_table *h, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                                       const double *delta, int64_t n_zeros, int n_weights, const int *weight_slots,
                                       double grid_half_width, int grid_steps, double *out_h_unpol,
                                       double *out_h_pol, double *out_ddy_pol) {
    const char *who = "mb_polish_peaks_weights";
    MB_CHECK_ARG(h && weight_slots && out_h_unpol && out_h_pol && out_ddy_pol, "%s: null argument", who);
    MB_CHECK_ARG(n_weights >= 1 && n_weights <= 64, "%s: n_weights=%d (1..64)", who, n_weights);
    MB_CHECK_ARG(P <= MAX_POLISH_PEAKS, "%s: P=%lld above %lld peaks per call", who, (long long)P,
                 (long long)MAX_POLISH_PEAKS);
    Table &t = table_of(h);
    MB_TRY(check_peaks(t, P, v_int, v_frac, delta, n_zeros, who));
    for (int w = 0; w < n_weights; ++w) MB_TRY(check_weights(t, weight_slots[w], who));
    MB_CHECK_ARG(grid_steps >= 0 && grid_steps <= (1 << 19) && std::isfinite(grid_half_width), "%s: bad grid", who);
    if (P == 0) return MB_OK;
    if (n_zeros == 0) {                                  // nothing to hold: the per-weight form
        for (int w = 0; w < n_weights; ++w)
            MB_TRY(mb_polish_peaks_exact(h, P, v_int, v_frac, delta, 0, weight_slots[w], grid_half_width,
                                         grid_steps, out_h_unpol + w * P, out_h_pol + w * P, out_ddy_pol + w * P));
        return MB_OK;
    }
    MB_TRY(device_guard(t.device));
    ExactStage s;
    MB_TRY(stage_exact(t, P, v_int, v_frac, delta, nullptr, 0, 0, s));
    // the matrices take at most AB_BUDGET bytes and at most half of the device's free memory
    size_t free_b = 0, total_b = 0;
    MB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t budget = std::min(AB_BUDGET, free_b / 2);
    const int64_t chunk =
        std::max<int64_t>(1, std::min<int64_t>({P, (int64_t)65535, (int64_t)(budget / (16 * (size_t)n_zeros))}));
    const size_t out_b = (size_t)n_weights * P * 8;
    DevBuf buf;
    MB_TRY(buf.ensure(2 * ((size_t)chunk * n_zeros * 8 + 256) + 3 * (out_b + 256)));
    char *q = (char *)buf.p;
    double *A = carve<double>(q, chunk * n_zeros);
    double *B = carve<double>(q, chunk * n_zeros);
    double *hu = carve<double>(q, (int64_t)n_weights * P);
    double *hp = carve<double>(q, (int64_t)n_weights * P);
    double *dp = carve<double>(q, (int64_t)n_weights * P);
    const ABExact ex{view(t), s.vi, s.vf, s.delta};
    cudaError_t e = cudaSuccess;
    for (int64_t c0 = 0; c0 < P && e == cudaSuccess; c0 += chunk) {
        const int64_t cn = std::min(chunk, P - c0);
        exact_ab_kernel<<<dim3((unsigned)((n_zeros + 255) / 256), (unsigned)cn), 256, 0, t.stream>>>(ex, n_zeros, c0,
                                                                                                     A, B);
        e = cudaGetLastError();
        for (int w = 0; w < n_weights && e == cudaSuccess; ++w) {
            const int64_t o = (int64_t)w * P + c0;
            PolishArgs a{n_zeros, t.d_gamma, t.d_weights[weight_slots[w]], nullptr, grid_steps, grid_half_width,
                         nullptr, hu + o, hp + o, dp + o};
            peak_polish_kernel<ABMatrix, POLISH_EVAL_FAST>
                <<<(unsigned)(cn * POLISH_CLUSTER), POLISH_THREADS, 0, t.stream>>>(ABMatrix{A, B, n_zeros}, a);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_h_unpol, hu, out_b, cudaMemcpyDeviceToHost, t.stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_h_pol, hp, out_b, cudaMemcpyDeviceToHost, t.stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_ddy_pol, dp, out_b, cudaMemcpyDeviceToHost, t.stream);
    const cudaError_t es = cudaStreamSynchronize(t.stream);       // nothing in flight before the free
    if (e == cudaSuccess) e = es;
    buf.release();
    if (e != cudaSuccess) {
        set_error("%s: %s", who, cudaGetErrorString(e));
        return MB_ERR_CUDA;
    }
    return MB_OK;
}

extern "C" int mb_fast_polish_exact(mb_table *h, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                                    const double *delta, int64_t n_zeros, int weight_slot, const double *ddy_grid,
                                    int64_t n_grid, int top, double *out_h_unpol, double *out_h_pol,
                                    double *out_ddy_pol) {
    const char *who = "mb_fast_polish_exact";
    MB_CHECK_ARG(h && out_h_unpol && out_h_pol && out_ddy_pol, "%s: null argument", who);
    MB_CHECK_ARG(P <= MAX_POLISH_PEAKS, "%s: P=%lld above %lld peaks per call", who, (long long)P,
                 (long long)MAX_POLISH_PEAKS);
    Table &t = table_of(h);
    MB_TRY(check_peaks(t, P, v_int, v_frac, delta, n_zeros, who));
    MB_TRY(check_weights(t, weight_slot, who));
    MB_TRY(check_grid(ddy_grid, n_grid, who));
    MB_CHECK_ARG(top >= 0 && top <= 65536, "%s: top=%d", who, top);
    if (P == 0) return MB_OK;
    MB_TRY(device_guard(t.device));
    const int nsel = (int)std::min<int64_t>(top, P);
    ExactStage s;
    MB_TRY(stage_exact(t, P, v_int, v_frac, delta, ddy_grid, n_grid, nsel, s));
    const ABExact src{view(t), s.vi, s.vf, s.delta};
    const double *d_w = t.d_weights[weight_slot];
    MomentArgs m{n_zeros, t.d_gamma, d_w, s.grid, (int)n_grid, s.hu, s.hp, s.dp};
    taylor_moments_kernel<ABExact><<<(unsigned)(P * POLISH_CLUSTER), POLISH_THREADS, 0, t.stream>>>(src, m);
    MB_CUDA(cudaGetLastError());
    MB_TRY(fetch_outputs(t.stream, P, s.hu, s.hp, s.dp, out_h_unpol, out_h_pol, out_ddy_pol));
    if (nsel == 0) return MB_OK;
    const std::vector<int> sel = top_indices(out_h_pol, P, nsel);
    MB_CUDA(cudaMemcpyAsync(s.sel, sel.data(), nsel * sizeof(int), cudaMemcpyHostToDevice, t.stream));
    PolishArgs a{n_zeros, t.d_gamma, d_w, nullptr, 0, 0.0, s.sel, s.hu, s.hp, s.dp};
    peak_polish_kernel<ABExact, POLISH_TOPK><<<(unsigned)(nsel * POLISH_CLUSTER), POLISH_THREADS, 0, t.stream>>>(src, a);
    MB_CUDA(cudaGetLastError());
    return fetch_outputs(t.stream, P, s.hu, s.hp, s.dp, out_h_unpol, out_h_pol, out_ddy_pol);
}
