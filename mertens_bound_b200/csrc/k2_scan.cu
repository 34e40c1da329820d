// Grid scan: K2 at y_m = v + m step for m = m0 .. m0 + n_m - 1 (search/polish.py:50-72 evaluates
// h(y0 + m step) the same way in FP64 from phi_j = gamma_j y0 mod 2pi and dphi_j = gamma_j step
// mod 2pi).  Here step is a 64.64 fixed-point number and the phase of every grid point is exact:
//   frac(y_m G) = frac(frac(v G) + m frac(step G))     (128-bit words, mod 1)
// Each thread takes MPT consecutive grid points: one 128 x 32-bit product per zero gives the
// exact phase of the first, whose sine/cosine (FP64, quarter-turn polynomials) times the
// amplitude is rotated to the other MPT - 1 points by powers of (cos, sin)(2 pi frac(step G)) of
// that zero (the reference's angle addition, polish.py:60-66, gpu_mertens_stream.cu:324-356,
// anchored afresh at an exact phase every MPT points; each point at most four rotations from its
// anchor).  FP64 accumulation, deterministic reduction over zero chunks.
#include <algorithm>
#include <cmath>

#include "k2_common.cuh"
#include "k2_internal.h"

namespace mb {
namespace {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_MPT = 16;                    // grid points per thread (one exact anchor)
static_assert(SCAN_MPT == 16, "add_rotations16 covers 16 points");
constexpr int SCAN_TILE = 256;                  // zeros per staged tile
struct __align__(16) ZScan {
    uint64_t p_lo, p_hi;       // frac(v G) + psi, 2^-128 units
    uint64_t d_lo, d_hi;       // frac(step G), 2^-128 units
    double a;                  // 2 |c| exp(-k gamma^2)
    double rc[4], rs[4];       // cos, sin of 2^b 2 pi frac(step G), b = 0..3
    double pad;
};

// (c, s) rotated by the angle whose cosine and sine are (cd, sd)
MB_DEV void rot(double c, double s, double cd, double sd, double &oc, double &os) {
    oc = fma(c, cd, -s * sd);
    os = fma(s, cd, c * sd);
}

// acc[i] += Re((c + i s) e^{i i phi}) for i = 0..15, given (rc[b], rs[b]) = (cos, sin)(2^b phi):
// a rotation tree of depth 4 (z8 from z0, z4 and z12, then the even points, then the odd ones,
// which need only their cosine), so every point is at most four rotations from the exact anchor
// and the chains are independent.
MB_DEV void add_rotations16(double c0, double s0, const double (&rc)[4], const double (&rs)[4], double (&acc)[16]) {
    double c[16], s[16];
    c[0] = c0;
    s[0] = s0;
    rot(c[0], s[0], rc[3], rs[3], c[8], s[8]);
#pragma unroll
    for (int i = 0; i < 16; i += 8) rot(c[i], s[i], rc[2], rs[2], c[i + 4], s[i + 4]);
#pragma unroll
    for (int i = 0; i < 16; i += 4) rot(c[i], s[i], rc[1], rs[1], c[i + 2], s[i + 2]);
#pragma unroll
    for (int i = 0; i < 16; i += 2) {
        acc[i] += c[i];
        acc[i + 1] += fma(c[i], rc[0], -s[i] * rs[0]);
    }
}

// (cos, sin)(2^b phi), b = 0..3, from (cos, sin)(phi) by repeated squaring
MB_DEV void rotation_powers(double cd, double sd, double (&rc)[4], double (&rs)[4]) {
    rc[0] = cd;
    rs[0] = sd;
#pragma unroll
    for (int b = 1; b < 4; ++b) {
        rc[b] = fma(rc[b - 1], rc[b - 1], -rs[b - 1] * rs[b - 1]);
        rs[b] = 2.0 * rc[b - 1] * rs[b - 1];
    }
}

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
            double cd, sd;
            sincospi(2.0 * s64_turns_to_f64(hi), &sd, &cd);   // ~1 ulp: errors add up over the rotations
            rotation_powers(cd, sd, r.rc, r.rs);
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
            const uint64_t xlo = z.p_lo + mlo;
            const uint64_t xhi = z.p_hi + mhi + (xlo < mlo ? 1 : 0);
            double sn, cs;
            sincos_turns_quad(s64_turns_to_f64(xhi), sn, cs);
            add_rotations16(cs * z.a, sn * z.a, z.rc, z.rs, acc);
        }
    }
    if (mb < n_m) {
        double *o = partial + ((int64_t)p * n_chunk + blockIdx.y) * n_m;
#pragma unroll
        for (int i = 0; i < SCAN_MPT; ++i)
            if (mb + i < n_m) o[mb + i] = acc[i];
    }
}

// Small grids over many base points (the hit polish of the enumerators): n_split CTAs per base
// point, each over a contiguous share of the zeros (so a few hits still fill the GPU), each thread
// HIT_ZPT zeros per round; the shares' sums go to partial[(p n_split + s) n_m + m] and
// hit_reduce_kernel adds them in split order.  Per zero: the exact phase at the grid's first point and
// the exact increment per step; every HIT_MB points an exact anchor (FP64 sine/cosine of the
// 128-bit phase, times the amplitude), rotated to the points in between by powers of the
// increment's (cos, sin).  A block of HIT_MB points is summed over the thread's zeros, then over
// the warp by a fixed shuffle tree, and lane 0 adds it to its warp's row of shared accumulators
// (fixed order -> deterministic).
constexpr int HIT_THREADS = 256;
constexpr int HIT_MAX_M = 1024;
constexpr int HIT_ZPT = 2;
constexpr int HIT_MB = 16;
static_assert(HIT_MB == 16, "add_rotations16 and the anchor step (increment << 4) assume 16");

__global__ void __launch_bounds__(HIT_THREADS)
k2_hit_scan_kernel(TabView t, const uint64_t *vi, const uint64_t *vf, uint64_t si, uint64_t sf, int64_t m0, int n_m,
                   int64_t n_use, double k, int n_split, double *partial) {
    extern __shared__ double acc[];            // [HIT_THREADS / 32][n_m]
    const int64_t p = blockIdx.x / n_split;
    const int split = blockIdx.x - (int)(p * n_split);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < (HIT_THREADS / 32) * n_m; i += HIT_THREADS) acc[i] = 0.0;
    __syncthreads();
    const uint64_t a_int = vi[p], a_frac = vf[p];
    const uint32_t mabs = (uint32_t)(m0 < 0 ? -m0 : m0);
    constexpr int PER_ROUND = HIT_THREADS * HIT_ZPT;
    const int64_t rounds = (n_use + PER_ROUND - 1) / PER_ROUND;
    const int64_t r_end = rounds * (split + 1) / n_split;
    for (int64_t r = rounds * split / n_split; r < r_end; ++r) {
        uint64_t xlo[HIT_ZPT], xhi[HIT_ZPT], dlo[HIT_ZPT], dhi[HIT_ZPT];
        double a[HIT_ZPT], rc[HIT_ZPT][4], rs[HIT_ZPT][4];
#pragma unroll
        for (int z = 0; z < HIT_ZPT; ++z) {
            const int64_t j = r * PER_ROUND + z * HIT_THREADS + threadIdx.x;
            xlo[z] = xhi[z] = dlo[z] = dhi[z] = 0;
            a[z] = 0.0;
            double cd = 1.0, sd = 0.0;
            if (j < n_use) {
                uint64_t hi, lo;
                phase128_exact((uint32_t)a_frac, (uint32_t)(a_frac >> 32), (uint32_t)a_int, (uint32_t)(a_int >> 32),
                               t.g0[j], t.g1[j], t.g2[j], t.g3[j], t.g4[j], hi, lo);
                const uint64_t plo = lo, phi = hi + t.psi[j];
                phase128_exact((uint32_t)sf, (uint32_t)(sf >> 32), (uint32_t)si, (uint32_t)(si >> 32), t.g0[j],
                               t.g1[j], t.g2[j], t.g3[j], t.g4[j], dhi[z], dlo[z]);
                uint64_t mlo = (uint64_t)mabs * dlo[z];
                uint64_t mhi = __umul64hi((uint64_t)mabs, dlo[z]) + (uint64_t)mabs * dhi[z];
                if (m0 < 0) {
                    mlo = ~mlo + 1;
                    mhi = ~mhi + (mlo == 0 ? 1 : 0);
                }
                xlo[z] = plo + mlo;
                xhi[z] = phi + mhi + (xlo[z] < mlo ? 1 : 0);
                const double g = t.gamma[j];
                a[z] = 2.0 * t.alpha[j] * exp(-k * g * g);
                sincospi(2.0 * s64_turns_to_f64(dhi[z]), &sd, &cd);   // ~1 ulp: errors add up over the rotations
                // the anchors advance by HIT_MB steps: d <<= log2(HIT_MB) (mod 2^128)
                dhi[z] = (dhi[z] << 4) | (dlo[z] >> 60);
                dlo[z] <<= 4;
            }
            rotation_powers(cd, sd, rc[z], rs[z]);
        }
        for (int mb = 0; mb < n_m; mb += HIT_MB) {
            double v[HIT_MB];
#pragma unroll
            for (int i = 0; i < HIT_MB; ++i) v[i] = 0.0;
#pragma unroll
            for (int z = 0; z < HIT_ZPT; ++z) {
                double sn, cs;
                sincos_turns_quad(s64_turns_to_f64(xhi[z]), sn, cs);
                add_rotations16(cs * a[z], sn * a[z], rc[z], rs[z], v);
                const uint64_t nlo = xlo[z] + dlo[z];
                xhi[z] = xhi[z] + dhi[z] + (nlo < xlo[z] ? 1 : 0);
                xlo[z] = nlo;
            }
#pragma unroll
            for (int i = 0; i < HIT_MB; ++i)
                for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
            if (lane == 0) {
#pragma unroll
                for (int i = 0; i < HIT_MB; ++i)
                    if (mb + i < n_m) acc[warp * n_m + mb + i] += v[i];
            }
        }
    }
    __syncthreads();
    for (int m = threadIdx.x; m < n_m; m += HIT_THREADS) {
        double s = 0.0;
        for (int w = 0; w < HIT_THREADS / 32; ++w) s += acc[w * n_m + m];
        partial[(int64_t)blockIdx.x * n_m + m] = s;
    }
}

__global__ void hit_reduce_kernel(const double *partial, int64_t P, int n_split, int n_m, double *h) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= P * n_m) return;
    const int64_t p = idx / n_m;
    const int m = (int)(idx - p * n_m);
    double s = 0.0;
    for (int c = 0; c < n_split; ++c) s += partial[(p * n_split + c) * n_m + m];
    h[idx] = s;
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
    // splits per hit: about 8 CTAs per SM in all, each split at least two rounds of zeros
    int sms = 148;
    MB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, t.device));
    const int64_t rounds = (n_use + HIT_THREADS * HIT_ZPT - 1) / (HIT_THREADS * HIT_ZPT);
    const int n_split = (int)std::max<int64_t>(1, std::min<int64_t>((8 * sms + P - 1) / P, rounds / 2));
    MB_TRY(t.work.ensure((size_t)P * n_split * n_m * sizeof(double)));
    double *partial = (double *)t.work.p;
    const size_t smem = (size_t)(HIT_THREADS / 32) * n_m * sizeof(double);
    if (smem > 48 * 1024)
        MB_CUDA(cudaFuncSetAttribute(k2_hit_scan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k2_hit_scan_kernel<<<(unsigned)(P * n_split), HIT_THREADS, smem, t.stream>>>(
        view(t), d_vi, d_vf, step_int, step_frac, m0, (int)n_m, n_use, k, n_split, partial);
    MB_CUDA(cudaGetLastError());
    hit_reduce_kernel<<<(unsigned)((P * n_m + 255) / 256), 256, 0, t.stream>>>(partial, P, n_split, (int)n_m, d_h);
    MB_CUDA(cudaGetLastError());
    MB_CUDA(cudaMemcpyAsync(out_h, d_h, hb, cudaMemcpyDeviceToHost, t.stream));
    MB_CUDA(cudaStreamSynchronize(t.stream));
    return MB_OK;
}
