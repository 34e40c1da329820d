// Grid scan: K2 at y_m = v + m step for m = m0 .. m0 + n_m - 1 (search/polish.py:50-72 evaluates
// h(y0 + m step) the same way in FP64 from phi_j = gamma_j y0 mod 2pi and dphi_j = gamma_j step
// mod 2pi).  Here step is a 64.64 fixed-point number and the phase of every grid point is exact:
//   frac(y_m G) = frac(frac(v G) + m frac(step G))     (128-bit words, mod 1)
// Each thread takes MPT consecutive grid points: one 128 x 32-bit product per zero gives the
// first, 128-bit additions give the rest.  Sine/cosine in FP64 (quarter-turn polynomials), FP64
// accumulation, deterministic reduction over zero chunks.
#include <algorithm>
#include <cmath>

#include "k2_common.cuh"
#include "k2_internal.h"

namespace mb {
namespace {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_MPT = 8;                     // grid points per thread
constexpr int SCAN_TILE = 256;                  // zeros per staged tile
struct __align__(16) ZScan {
    uint64_t p_lo, p_hi;       // frac(v G) + psi, 2^-128 units
    uint64_t d_lo, d_hi;       // frac(step G), 2^-128 units
    double a;                  // 2 |c| exp(-k gamma^2)
    double pad;
};

// partial[((p * n_chunk) + chunk) * n_m + m]
__global__ void __launch_bounds__(SCAN_THREADS)
k2_scan_kernel(TabView t, const uint64_t *vi, const uint64_t *vf, uint64_t si, uint64_t sf, int64_t m0, int n_m,
               int64_t n_use, int64_t chunk, double k, double *partial) {
    __shared__ ZScan tile[SCAN_TILE];
    const int p = blockIdx.z;
    const int n_chunk = gridDim.y;
    const int mb = (blockIdx.x * SCAN_THREADS + threadIdx.x) * SCAN_MPT;     // first local grid index
    const uint64_t a_int = vi[p], a_frac = vf[p];
    double acc[SCAN_MPT];
#pragma unroll
    for (int i = 0; i < SCAN_MPT; ++i) acc[i] = 0.0;
    const int64_t z0 = (int64_t)blockIdx.y * chunk, z1 = min(z0 + chunk, n_use);
    const int64_t mstart = m0 + mb;                       // signed grid index of this thread's first point
    const uint32_t mabs = (uint32_t)(mstart < 0 ? -mstart : mstart);
    for (int64_t tb = z0; tb < z1; tb += SCAN_TILE) {
        __syncthreads();
        const int64_t j = tb + threadIdx.x;
        if (threadIdx.x < SCAN_TILE && j < z1) {
            ZScan r;
            uint64_t hi, lo;
            phase128_exact((uint32_t)a_frac, (uint32_t)(a_frac >> 32), (uint32_t)a_int, (uint32_t)(a_int >> 32),
                           t.g0[j], t.g1[j], t.g2[j], t.g3[j], t.g4[j], hi, lo);
            r.p_lo = lo;
            r.p_hi = hi + t.psi[j];
            phase128_exact((uint32_t)sf, (uint32_t)(sf >> 32), (uint32_t)si, (uint32_t)(si >> 32), t.g0[j], t.g1[j],
                           t.g2[j], t.g3[j], t.g4[j], hi, lo);
            r.d_lo = lo;
            r.d_hi = hi;
            const double g = t.gamma[j];
            r.a = 2.0 * t.alpha[j] * exp(-k * g * g);
            r.pad = 0.0;
            tile[threadIdx.x] = r;
        }
        __syncthreads();
        if (mb >= n_m) continue;
        const int nt = (int)min((int64_t)SCAN_TILE, z1 - tb);
        for (int jj = 0; jj < nt; ++jj) {
            const ZScan z = tile[jj];
            // x = p + mstart d  (mod 2^128)
            uint64_t mlo = (uint64_t)mabs * z.d_lo;
            uint64_t mhi = __umul64hi((uint64_t)mabs, z.d_lo) + (uint64_t)mabs * z.d_hi;
            if (mstart < 0) {                          // negate (two's complement, 128 bits)
                mlo = ~mlo + 1;
                mhi = ~mhi + (mlo == 0 ? 1 : 0);
            }
            uint64_t xlo = z.p_lo + mlo;
            uint64_t xhi = z.p_hi + mhi + (xlo < mlo ? 1 : 0);
#pragma unroll
            for (int i = 0; i < SCAN_MPT; ++i) {
                const double y = s64_turns_to_f64(xhi);
                double sn, cs;
                sincos_turns_quad(y, sn, cs);
                acc[i] = fma(z.a, cs, acc[i]);
                const uint64_t nlo = xlo + z.d_lo;
                xhi = xhi + z.d_hi + (nlo < xlo ? 1 : 0);
                xlo = nlo;
            }
        }
    }
    if (mb < n_m) {
        double *o = partial + ((int64_t)p * n_chunk + blockIdx.y) * n_m;
#pragma unroll
        for (int i = 0; i < SCAN_MPT; ++i)
            if (mb + i < n_m) o[mb + i] = acc[i];
    }
}

// Small grids over many base points (the hit polish of the enumerators): one CTA per base point,
// threads over zeros; for each zero the exact phase at the base point and the exact increment
// per grid step, then every grid point in turn: warp-shuffle sum of the 32 lanes' terms, added
// by lane 0 to its warp's row of shared accumulators (fixed order -> deterministic).
constexpr int HIT_THREADS = 256;
constexpr int HIT_MAX_M = 1024;

__global__ void __launch_bounds__(HIT_THREADS)
k2_hit_scan_kernel(TabView t, const uint64_t *vi, const uint64_t *vf, uint64_t si, uint64_t sf, int64_t m0, int n_m,
                   int64_t n_use, double k, double *out_h) {
    extern __shared__ double acc[];            // [HIT_THREADS / 32][n_m]
    const int p = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < (HIT_THREADS / 32) * n_m; i += HIT_THREADS) acc[i] = 0.0;
    __syncthreads();
    const uint64_t a_int = vi[p], a_frac = vf[p];
    const uint32_t mabs = (uint32_t)(m0 < 0 ? -m0 : m0);
    const int64_t rounds = (n_use + HIT_THREADS - 1) / HIT_THREADS;
    for (int64_t r = 0; r < rounds; ++r) {
        const int64_t j = r * HIT_THREADS + threadIdx.x;
        const bool live = j < n_use;
        uint64_t xlo = 0, xhi = 0, dlo = 0, dhi = 0;
        double a = 0.0;
        if (live) {
            uint64_t hi, lo;
            phase128_exact((uint32_t)a_frac, (uint32_t)(a_frac >> 32), (uint32_t)a_int, (uint32_t)(a_int >> 32),
                           t.g0[j], t.g1[j], t.g2[j], t.g3[j], t.g4[j], hi, lo);
            const uint64_t plo = lo, phi = hi + t.psi[j];
            phase128_exact((uint32_t)sf, (uint32_t)(sf >> 32), (uint32_t)si, (uint32_t)(si >> 32), t.g0[j], t.g1[j],
                           t.g2[j], t.g3[j], t.g4[j], dhi, dlo);
            uint64_t mlo = (uint64_t)mabs * dlo;
            uint64_t mhi = __umul64hi((uint64_t)mabs, dlo) + (uint64_t)mabs * dhi;
            if (m0 < 0) {
                mlo = ~mlo + 1;
                mhi = ~mhi + (mlo == 0 ? 1 : 0);
            }
            xlo = plo + mlo;
            xhi = phi + mhi + (xlo < mlo ? 1 : 0);
            const double g = t.gamma[j];
            a = 2.0 * t.alpha[j] * exp(-k * g * g);
        }
        for (int m = 0; m < n_m; ++m) {
            double v = 0.0;
            if (live) {
                double sn, cs;
                sincos_turns_quad(s64_turns_to_f64(xhi), sn, cs);
                v = a * cs;
                const uint64_t nlo = xlo + dlo;
                xhi = xhi + dhi + (nlo < xlo ? 1 : 0);
                xlo = nlo;
            }
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) acc[warp * n_m + m] += v;
        }
    }
    __syncthreads();
    for (int m = threadIdx.x; m < n_m; m += HIT_THREADS) {
        double s = 0.0;
        for (int w = 0; w < HIT_THREADS / 32; ++w) s += acc[w * n_m + m];
        out_h[(int64_t)p * n_m + m] = s;
    }
}

__global__ void scan_reduce_kernel(const double *partial, int P, int n_chunk, int n_m, double *h) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)P * n_m) return;
    const int p = (int)(idx / n_m), m = (int)(idx - (int64_t)p * n_m);
    double s = 0.0;
    for (int c = 0; c < n_chunk; ++c) s += partial[((int64_t)p * n_chunk + c) * n_m + m];
    h[idx] = s;
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" int mb_grid_scan(mb_table *h, int64_t P, const uint64_t *v_int, const uint64_t *v_frac, double k,
                            double T, uint64_t step_int, uint64_t step_frac, int64_t m0, int64_t n_m, double *out_h) {
    MB_CHECK_ARG(h && v_int && v_frac && out_h, "mb_grid_scan: null argument");
    MB_CHECK_ARG(P >= 0 && P <= 65535, "mb_grid_scan: P=%lld (0..65535)", (long long)P);
    MB_CHECK_ARG(n_m >= 0 && n_m <= (1 << 26) && P * n_m <= ((int64_t)1 << 28), "mb_grid_scan: n_m=%lld", (long long)n_m);
    MB_CHECK_ARG(m0 > -((int64_t)1 << 31) && m0 + n_m < ((int64_t)1 << 31), "mb_grid_scan: grid indices exceed 2^31");
    MB_CHECK_ARG(std::isfinite(k) && k >= 0.0 && !std::isnan(T), "mb_grid_scan: bad k or T");
    if (P == 0 || n_m == 0) return MB_OK;
    Table &t = table_of(h);
    MB_TRY(device_guard(t.device));
    const int64_t n_use = t.count_below(T);
    const size_t cb = (size_t)P * 8, hb = (size_t)P * n_m * 8;
    int sms = 148;
    MB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, t.device));
    const int64_t per_cta = (int64_t)SCAN_THREADS * SCAN_MPT;
    const int64_t n_mt = (n_m + per_cta - 1) / per_cta;
    int64_t n_chunk = std::max<int64_t>(1, ((int64_t)sms * 4 + n_mt * P - 1) / (n_mt * P));
    n_chunk = std::min<int64_t>(n_chunk, std::max<int64_t>(1, (n_use + SCAN_TILE - 1) / SCAN_TILE));
    int64_t chunk = std::max<int64_t>(SCAN_TILE, ((n_use + n_chunk - 1) / n_chunk + SCAN_TILE - 1) / SCAN_TILE * SCAN_TILE);
    n_chunk = std::max<int64_t>(1, (n_use + chunk - 1) / chunk);
    MB_TRY(t.io.ensure(2 * cb + hb + 256));
    MB_TRY(t.work.ensure((size_t)P * n_chunk * n_m * 8));
    char *base = (char *)t.io.p;
    uint64_t *d_vi = (uint64_t *)base, *d_vf = (uint64_t *)(base + cb);
    double *d_h = (double *)(base + ((2 * cb + 255) & ~(size_t)255));
    double *partial = (double *)t.work.p;
    MB_CUDA(cudaMemcpyAsync(d_vi, v_int, cb, cudaMemcpyHostToDevice, t.stream));
    MB_CUDA(cudaMemcpyAsync(d_vf, v_frac, cb, cudaMemcpyHostToDevice, t.stream));
    if (n_use == 0) {
        MB_CUDA(cudaMemsetAsync(partial, 0, (size_t)P * n_m * 8, t.stream));
        n_chunk = 1;
    } else {
        dim3 grid((unsigned)n_mt, (unsigned)n_chunk, (unsigned)P);
        k2_scan_kernel<<<grid, SCAN_THREADS, 0, t.stream>>>(view(t), d_vi, d_vf, step_int, step_frac, m0, (int)n_m,
                                                            n_use, chunk, k, partial);
        MB_CUDA(cudaGetLastError());
    }
    const int64_t total = P * n_m;
    scan_reduce_kernel<<<(unsigned)((total + 255) / 256), 256, 0, t.stream>>>(partial, (int)P, (int)n_chunk, (int)n_m, d_h);
    MB_CUDA(cudaGetLastError());
    MB_CUDA(cudaMemcpyAsync(out_h, d_h, hb, cudaMemcpyDeviceToHost, t.stream));
    MB_CUDA(cudaStreamSynchronize(t.stream));
    return MB_OK;
}

extern "C" int mb_hit_scan(mb_table *h, int64_t P, const uint64_t *v_int, const uint64_t *v_frac, double k,
                           int64_t n_use, uint64_t step_int, uint64_t step_frac, int64_t m0, int64_t n_m,
                           double *out_h) {
    MB_CHECK_ARG(h && v_int && v_frac && out_h, "mb_hit_scan: null argument");
    MB_CHECK_ARG(P >= 0 && P <= (1 << 24), "mb_hit_scan: P=%lld", (long long)P);
    MB_CHECK_ARG(n_m >= 1 && n_m <= HIT_MAX_M, "mb_hit_scan: n_m=%lld (1..%d)", (long long)n_m, HIT_MAX_M);
    MB_CHECK_ARG(m0 > -((int64_t)1 << 31) && m0 + n_m < ((int64_t)1 << 31), "mb_hit_scan: grid indices exceed 2^31");
    MB_CHECK_ARG(std::isfinite(k) && k >= 0.0, "mb_hit_scan: k=%g", k);
    if (P == 0) return MB_OK;
    Table &t = table_of(h);
    MB_CHECK_ARG(n_use >= 0 && n_use <= t.n, "mb_hit_scan: n_use=%lld of %lld", (long long)n_use, (long long)t.n);
    MB_TRY(device_guard(t.device));
    const size_t cb = (size_t)P * 8, hb = (size_t)P * n_m * 8;
    MB_TRY(t.io.ensure(2 * cb + hb + 256));
    char *base = (char *)t.io.p;
    uint64_t *d_vi = (uint64_t *)base, *d_vf = (uint64_t *)(base + cb);
    double *d_h = (double *)(base + ((2 * cb + 255) & ~(size_t)255));
    MB_CUDA(cudaMemcpyAsync(d_vi, v_int, cb, cudaMemcpyHostToDevice, t.stream));
    MB_CUDA(cudaMemcpyAsync(d_vf, v_frac, cb, cudaMemcpyHostToDevice, t.stream));
    const size_t smem = (size_t)(HIT_THREADS / 32) * n_m * sizeof(double);
    if (smem > 48 * 1024)
        MB_CUDA(cudaFuncSetAttribute(k2_hit_scan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k2_hit_scan_kernel<<<(unsigned)P, HIT_THREADS, smem, t.stream>>>(view(t), d_vi, d_vf, step_int, step_frac, m0,
                                                                      (int)n_m, n_use, k, d_h);
    MB_CUDA(cudaGetLastError());
    MB_CUDA(cudaMemcpyAsync(out_h, d_h, hb, cudaMemcpyDeviceToHost, t.stream));
    MB_CUDA(cudaStreamSynchronize(t.stream));
    return MB_OK;
}
