// Drop-in replacements for the reference's C-ABI evaluator (search/path1_eval_fast.cpp),
// same names, argument meaning and host-array contract, computed on the current CUDA device:
//   compute_peak_AB            (:15-53)  x = y 2^30 as u128, xh = x >> 48, xl = x mod 2^48,
//                                        ph = xh ghi + xl glo - psi (mod 2^128), top 64 bits,
//                                        th = top64 2pi/2^64 + gamma dy0, A = 2 alpha cos th,
//                                        B = 2 alpha sin th  (P x N row-major outputs)
//   polish_peaks_with_weights  (:58-143) per peak: h0 = sum w A; grid of 2 grid_steps + 1 shifts
//                                        over the first min(N, 4096) zeros; <= 6 Newton steps on
//                                        ddy (clamp 1e-4, stop below 1e-13 or |f''| <= 1e-12);
//                                        keep the larger |h|.
// The reference functions return void and check nothing.  Here the mb_* forms return a status;
// the void forms print the error to stderr and fill their outputs with NaN, so a failure is
// never silent.  A/B are the reference's contract (HBM- and transfer-bound); the fused mb_k2_*
// entry points are the fast path.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>

#include "k2_internal.h"
#include "k2_polish.cuh"

namespace mb {
namespace {

struct Uint128 {
    uint64_t lo, hi;
};

__device__ __forceinline__ Uint128 mul64x128_mod(uint64_t a, uint64_t blo, uint64_t bhi) {
    Uint128 r;
    r.lo = a * blo;
    r.hi = __umul64hi(a, blo) + a * bhi;
    return r;
}

__global__ void peak_AB_kernel(int n_peaks, int n_zeros, const uint64_t *x_lo, const uint64_t *x_hi,
                               const double *dy0, const double *alpha, const double *gamma,
                               const uint64_t *ghi_lo, const uint64_t *ghi_hi, const uint64_t *glo_lo,
                               const uint64_t *glo_hi, const uint64_t *psi_lo, const uint64_t *psi_hi,
                               double *A, double *B) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int p = blockIdx.y;
    if (i >= n_zeros || p >= n_peaks) return;
    const uint64_t xl0 = x_lo[p], xh0 = x_hi[p];
    const uint64_t xh = (xl0 >> 48) | (xh0 << 16);          // (uint64_t)(x >> 48)
    const uint64_t xl = xl0 & ((1ull << 48) - 1);
    const Uint128 a = mul64x128_mod(xh, ghi_lo[i], ghi_hi[i]);
    const Uint128 b = mul64x128_mod(xl, glo_lo[i], glo_hi[i]);
    uint64_t lo = a.lo + b.lo;
    uint64_t hi = a.hi + b.hi + (lo < a.lo ? 1 : 0);
    const uint64_t plo = psi_lo[i];
    hi = hi - psi_hi[i] - (lo < plo ? 1 : 0);
    lo = lo - plo;
    const double scale = 2.0 * 3.14159265358979323846 * 5.421010862427522e-20;
    const double th = (double)hi * scale + gamma[i] * dy0[p];
    double s, c;
    sincos(th, &s, &c);
    const double ta = 2.0 * alpha[i];
    const size_t o = (size_t)p * n_zeros + i;
    A[o] = ta * c;
    B[o] = ta * s;
}

}  // namespace

// Per-device grow-only buffers of the handle-free entry points (the reference API has no handle).
struct ScratchState {
    std::mutex mu;
    DevBuf buf[64];
};
static ScratchState g_scratch;

std::mutex &scratch_mutex() { return g_scratch.mu; }

int scratch_buffer(size_t bytes, void **out) {
    int dev = 0;
    MB_CUDA(cudaGetDevice(&dev));
    MB_CHECK_ARG(dev >= 0 && dev < 64, "scratch: device %d", dev);
    MB_TRY(g_scratch.buf[dev].ensure(bytes));
    *out = g_scratch.buf[dev].p;
    return MB_OK;
}

}  // namespace mb

using namespace mb;

extern "C" int mb_compute_peak_AB(int n_peaks, const uint64_t *x_lo_arr, const uint64_t *x_hi_arr,
                                  const double *dy0_arr, int n_zeros, const double *alpha, const double *gamma,
                                  const uint64_t *ghi_lo, const uint64_t *ghi_hi, const uint64_t *glo_lo,
                                  const uint64_t *glo_hi, const uint64_t *psi_lo, const uint64_t *psi_hi,
                                  double *out_A, double *out_B) {
    MB_CHECK_ARG(n_peaks >= 0 && n_zeros >= 0, "compute_peak_AB: negative size");
    if (n_peaks == 0 || n_zeros == 0) return MB_OK;
    MB_CHECK_ARG(x_lo_arr && x_hi_arr && dy0_arr && alpha && gamma && ghi_lo && ghi_hi && glo_lo && glo_hi &&
                 psi_lo && psi_hi && out_A && out_B, "compute_peak_AB: null array");
    std::lock_guard<std::mutex> lock(scratch_mutex());
    const size_t N = (size_t)n_zeros;
    // peaks per pass so that the A/B slabs stay within 2 GiB of device memory
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)n_peaks, ((size_t)1 << 31) / (16 * N)));
    const size_t bytes = 8 * (N * 8 + 256) + 3 * ((size_t)chunk * 8 + 256) + 2 * ((size_t)chunk * N * 8 + 256);
    void *base = nullptr;
    MB_TRY(scratch_buffer(bytes, &base));
    char *p = (char *)base;
    double *d_alpha = carve<double>(p, N), *d_gamma = carve<double>(p, N);
    uint64_t *d_ghl = carve<uint64_t>(p, N), *d_ghh = carve<uint64_t>(p, N), *d_gll = carve<uint64_t>(p, N),
             *d_glh = carve<uint64_t>(p, N), *d_psl = carve<uint64_t>(p, N), *d_psh = carve<uint64_t>(p, N);
    uint64_t *d_xl = carve<uint64_t>(p, chunk), *d_xh = carve<uint64_t>(p, chunk);
    double *d_dy = carve<double>(p, chunk);
    double *d_A = carve<double>(p, (size_t)chunk * N), *d_B = carve<double>(p, (size_t)chunk * N);
    cudaStream_t s = cudaStreamPerThread;
    MB_CUDA(cudaMemcpyAsync(d_alpha, alpha, N * 8, cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaMemcpyAsync(d_gamma, gamma, N * 8, cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaMemcpyAsync(d_ghl, ghi_lo, N * 8, cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaMemcpyAsync(d_ghh, ghi_hi, N * 8, cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaMemcpyAsync(d_gll, glo_lo, N * 8, cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaMemcpyAsync(d_glh, glo_hi, N * 8, cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaMemcpyAsync(d_psl, psi_lo, N * 8, cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaMemcpyAsync(d_psh, psi_hi, N * 8, cudaMemcpyHostToDevice, s));
    for (int p0 = 0; p0 < n_peaks; p0 += chunk) {
        const int np = std::min(chunk, n_peaks - p0);
        MB_CUDA(cudaMemcpyAsync(d_xl, x_lo_arr + p0, np * 8, cudaMemcpyHostToDevice, s));
        MB_CUDA(cudaMemcpyAsync(d_xh, x_hi_arr + p0, np * 8, cudaMemcpyHostToDevice, s));
        MB_CUDA(cudaMemcpyAsync(d_dy, dy0_arr + p0, np * 8, cudaMemcpyHostToDevice, s));
        dim3 grid((unsigned)((N + 255) / 256), (unsigned)np);
        peak_AB_kernel<<<grid, 256, 0, s>>>(np, n_zeros, d_xl, d_xh, d_dy, d_alpha, d_gamma, d_ghl, d_ghh, d_gll,
                                            d_glh, d_psl, d_psh, d_A, d_B);
        MB_CUDA(cudaGetLastError());
        MB_CUDA(cudaMemcpyAsync(out_A + (size_t)p0 * N, d_A, (size_t)np * N * 8, cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaMemcpyAsync(out_B + (size_t)p0 * N, d_B, (size_t)np * N * 8, cudaMemcpyDeviceToHost, s));
    }
    MB_CUDA(cudaStreamSynchronize(s));
    return MB_OK;
}

extern "C" int mb_polish_peaks_with_weights(int n_peaks, int n_zeros, const double *A, const double *B,
                                            const double *gamma, const double *w, double grid_half_width,
                                            int grid_steps, double *out_h_unpol, double *out_h_pol,
                                            double *out_ddy_pol) {
    MB_CHECK_ARG(n_peaks >= 0 && n_zeros >= 0 && grid_steps >= 0, "polish_peaks_with_weights: negative size");
    if (n_peaks == 0) return MB_OK;
    MB_CHECK_ARG(A && B && gamma && w && out_h_unpol && out_h_pol && out_ddy_pol,
                 "polish_peaks_with_weights: null array");
    MB_CHECK_ARG(std::isfinite(grid_half_width), "polish_peaks_with_weights: grid_half_width is not finite");
    std::lock_guard<std::mutex> lock(scratch_mutex());
    const size_t N = (size_t)std::max(n_zeros, 1);
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)n_peaks, ((size_t)1 << 31) / (16 * N)));
    const size_t bytes = 2 * (N * 8 + 256) + 2 * ((size_t)chunk * N * 8 + 256) + 3 * ((size_t)chunk * 8 + 256);
    void *base = nullptr;
    MB_TRY(scratch_buffer(bytes, &base));
    char *p = (char *)base;
    double *d_g = carve<double>(p, N), *d_w = carve<double>(p, N);
    double *d_A = carve<double>(p, (size_t)chunk * N), *d_B = carve<double>(p, (size_t)chunk * N);
    double *d_hu = carve<double>(p, chunk), *d_hp = carve<double>(p, chunk), *d_dp = carve<double>(p, chunk);
    cudaStream_t s = cudaStreamPerThread;
    if (n_zeros > 0) {
        MB_CUDA(cudaMemcpyAsync(d_g, gamma, (size_t)n_zeros * 8, cudaMemcpyHostToDevice, s));
        MB_CUDA(cudaMemcpyAsync(d_w, w, (size_t)n_zeros * 8, cudaMemcpyHostToDevice, s));
    }
    for (int p0 = 0; p0 < n_peaks; p0 += chunk) {
        const int np = std::min(chunk, n_peaks - p0);
        if (n_zeros > 0) {
            MB_CUDA(cudaMemcpyAsync(d_A, A + (size_t)p0 * n_zeros, (size_t)np * n_zeros * 8, cudaMemcpyHostToDevice, s));
            MB_CUDA(cudaMemcpyAsync(d_B, B + (size_t)p0 * n_zeros, (size_t)np * n_zeros * 8, cudaMemcpyHostToDevice, s));
        }
        PolishArgs a{n_zeros, d_g, d_w, nullptr, grid_steps, grid_half_width, nullptr, d_hu, d_hp, d_dp};
        peak_polish_kernel<ABMatrix, POLISH_EVAL_FAST><<<(unsigned)(np * POLISH_CLUSTER), POLISH_THREADS, 0, s>>>(ABMatrix{d_A, d_B, n_zeros}, a);
        MB_CUDA(cudaGetLastError());
        MB_CUDA(cudaMemcpyAsync(out_h_unpol + p0, d_hu, np * 8, cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaMemcpyAsync(out_h_pol + p0, d_hp, np * 8, cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaMemcpyAsync(out_ddy_pol + p0, d_dp, np * 8, cudaMemcpyDeviceToHost, s));
    }
    MB_CUDA(cudaStreamSynchronize(s));
    return MB_OK;
}

static void fill_nan(double *a, size_t n) {
    if (!a) return;
    for (size_t i = 0; i < n; ++i) a[i] = NAN;
}

extern "C" void compute_peak_AB(int n_peaks, const uint64_t *x_lo_arr, const uint64_t *x_hi_arr,
                                const double *dy0_arr, int n_zeros, const double *alpha, const double *gamma,
                                const uint64_t *ghi_lo, const uint64_t *ghi_hi, const uint64_t *glo_lo,
                                const uint64_t *glo_hi, const uint64_t *psi_lo, const uint64_t *psi_hi,
                                double *out_A, double *out_B) {
    int st = mb_compute_peak_AB(n_peaks, x_lo_arr, x_hi_arr, dy0_arr, n_zeros, alpha, gamma, ghi_lo, ghi_hi,
                                glo_lo, glo_hi, psi_lo, psi_hi, out_A, out_B);
    if (st != MB_OK) {
        fprintf(stderr, "compute_peak_AB failed: %s\n", mb::last_error());
        if (n_peaks > 0 && n_zeros > 0) {
            fill_nan(out_A, (size_t)n_peaks * n_zeros);
            fill_nan(out_B, (size_t)n_peaks * n_zeros);
        }
    }
}

extern "C" void polish_peaks_with_weights(int n_peaks, int n_zeros, const double *A, const double *B,
                                          const double *gamma, const double *w, double grid_half_width,
                                          int grid_steps, double *out_h_unpol, double *out_h_pol,
                                          double *out_ddy_pol) {
    int st = mb_polish_peaks_with_weights(n_peaks, n_zeros, A, B, gamma, w, grid_half_width, grid_steps,
                                          out_h_unpol, out_h_pol, out_ddy_pol);
    if (st != MB_OK) {
        fprintf(stderr, "polish_peaks_with_weights failed: %s\n", mb::last_error());
        if (n_peaks > 0) {
            fill_nan(out_h_unpol, n_peaks);
            fill_nan(out_h_pol, n_peaks);
            fill_nan(out_ddy_pol, n_peaks);
        }
    }
}
