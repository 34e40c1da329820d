// The chosen form: batched, precision-tiered K2 value + gradient.
//
// Each group (k, T, a range of candidates) splits its zeros [0, n_T) at a boundary n_h chosen
// from an a-priori error bound (host, k2_plan.cu):
//   heavy tier  j <  n_h : 64-bit phase (3 IMAD.lo + 4 DFMA + 4 FFMA, error ~2^-48 turn), sin/cos
//                          from a 2048-entry table rotated by short FP64 polynomials, FP64
//                          accumulation.                                  -> k2_heavy_kernel
//   light tier  j >= n_h : 32-bit phase (3 IMAD.lo + 4 DFMA in two chains; 2 IMAD.lo + 3 DFMA
//                          when every zero has gamma < 3.29e6, light_phase32_fused), MUFU sin/cos
//                          of the reduced phase, FP32 accumulation flushed every LIGHT_FLUSH terms
//                          into FP64 partials.                           -> k2_light_kernel
// The heavy kernel is persistent with two CTAs per SM (FP64-pipe bound); the light kernel is
// launched concurrently on a second stream with one CTA per work item and takes each SM as the
// heavy CTAs retire (XU / FMA / integer pipes), so the tiers overlap.
//
// Phase algebra (v = a1 2^32 + a0 + (d1 2^-32 + d0 2^-64), G = gI + b1 2^-32 + b0 2^-64 +
// c1 2^-96 + c0 2^-128, all limbs 32-bit):
//   frac(vG) 2^32 = [a1 b0 + a0 b1 + d1 gI]                       (exact mod 2^32, IMAD.lo)
//                 + (a0 b0 + a1 c1 + d0 gI + d1 b1) 2^-32           (< 2^34, FP64)
//                 + (a1 c0 + a0 c1 + d1 b0 + d0 b1) 2^-64 + ...     (< 4 units)
// The FP64 sums are formed on top of 1.5 2^52, so each DFMA rounds to an integer and the low
// mantissa words hold them mod 2^32 (error <= 2 units of 2^-32 turn; k2_light.cuh).
// arg(c)/2pi (psi) is added to the phase, so each term is a cos(2pi u) with a = 2|c| w.
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "k2_common.cuh"
#include "k2_fast.h"
#include "k2_internal.h"
#include "k2_light.cuh"

namespace mb {


struct __align__(16) ZLight {   // 64 B
    uint32_t b0, b1, gi, psi32;  // psi32 = round(psi 2^32) + 2 (centres the truncation bias)
    double b0s, c1s, gis, b1s;   // limb 2^-32 (exact)
    float a, b, d, pad;          // a = 2|c|w, b = -a gamma, d = -a gamma^2
};

struct __align__(16) ZLightF {  // 48 B: the light record of light_phase32_fused
    uint32_t b0, b1, psi32;      // as in ZLight, psi32 = round(psi 2^32) + 1
    float a;                     // a = 2|c|w
    double b0s, c1s;             // limb 2^-32 (exact)
    double gh;                   // gI 2^32 + b1 (exact for gI < 2^19)
    float b, d;                  // b = -a gamma, d = -a gamma^2
};

struct __align__(16) ZHeavy {   // 96 B
    uint32_t b0, b1, gi, psi_hi; // psi_hi = top 32 bits of arg(c)/2pi 2^64, plus 2^20 (half a table step)
    double b0s, c1s, gis, b1s;   // limb 2^-32
    float c0f, c1f, b0f, b1f;    // limb 2^-64 (FP32: these products need 2^-18 relative)
    float psi_lo, pad0;          // low 32 bits of arg(c)/2pi 2^64, times 2^-32
    double a, b, d;
};

constexpr int FAST_THREADS = 256;
constexpr int LIGHT_TILE = 256;
constexpr int HEAVY_TILE = 128;
constexpr int LIGHT_FLUSH = 32;
// shared memory: the staged tile, reused after the tile loop for the cross-warp reduction
constexpr int FAST_SMEM = 24576;
static_assert(FAST_SMEM >= LIGHT_TILE * sizeof(ZLight), "light tile");
static_assert(sizeof(ZLightF) == 48, "fused light record");
static_assert(FAST_SMEM >= HEAVY_TILE * sizeof(ZHeavy), "heavy tile");
static_assert(FAST_SMEM >= FAST_THREADS * 4 * 3 * sizeof(double), "reduction buffer");

// The angle 2pi u 2^-32 of a light term in radians: u (the signed phase in units of 2^-32 turn)
// converted to float, times fl_down(2pi) 2^-32 -- rounded down so that |th| <= 2^31 C =
// 3.14159250 < pi for every u, inside the range where __sinf / __cosf have their documented error
// bounds.  (A conversion-free form -- the bits 0x4B400000 + (u >> 9) as a float and one FFMA --
// measured 1-3% slower: the kernel is latency-bound, not XU-bound, and its chain is longer.)
constexpr float LIGHT_ANG_C = 6.2831850051879883f * 2.3283064365386963e-10f;   // fl_down(2pi) 2^-32
MB_DEV float light_angle(int32_t u) { return (float)u * LIGHT_ANG_C; }

template <int CPT, bool FUSED>
MB_DEV void light_tile(const void *tile_v, int nt, int zl, int ZL, const CandRegs (&cr)[CPT],
                       double (&sum)[CPT][3]) {
    using Rec = typename std::conditional<FUSED, ZLightF, ZLight>::type;
    const Rec *tile = static_cast<const Rec *>(tile_v);
    float acc[CPT][3];
#pragma unroll
    for (int i = 0; i < CPT; ++i) acc[i][0] = acc[i][1] = acc[i][2] = 0.f;
    // one zero's terms for every candidate of the thread
    auto term = [&](int jj) {
        const Rec z = tile[jj];
#pragma unroll
        for (int i = 0; i < CPT; ++i) {
            int32_t u;
            if constexpr (FUSED)
                u = (int32_t)light_phase32_fused(cr[i], z.b0, z.b1, z.b0s, z.c1s, z.gh, z.psi32);
            else
                u = (int32_t)light_phase32(cr[i], z.b0, z.b1, z.gi, z.b0s, z.c1s, z.gis, z.b1s, z.psi32);
            const float th = light_angle(u);
            float s = __sinf(th), co = __cosf(th);
            acc[i][0] = fmaf(z.a, co, acc[i][0]);
            acc[i][1] = fmaf(z.b, s, acc[i][1]);
            acc[i][2] = fmaf(z.d, co, acc[i][2]);
        }
    };
    auto flush = [&]() {
#pragma unroll
        for (int i = 0; i < CPT; ++i)
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                sum[i][q] += (double)acc[i][q];
                acc[i][q] = 0.f;
            }
    };
    // whole groups of LIGHT_FLUSH zeros (a fixed trip count, no per-zero counter), then the rest
    int jj = zl;
    for (; jj + (LIGHT_FLUSH - 1) * ZL < nt; jj += LIGHT_FLUSH * ZL) {
#pragma unroll 1
        for (int q = 0; q < LIGHT_FLUSH; ++q) term(jj + q * ZL);
        flush();
    }
    for (; jj < nt; jj += ZL) term(jj);
    flush();
}

// sin/cos(2 pi (q/2048 + r)) for |r| <= 2^-12 turn: the table entry (cos, sin)(2 pi q/2048)
// rotated by r: sin(2 pi r) = r (2pi - (2pi)^3 r^2 / 6) (truncation 7e-17) and
// cos(2 pi r) - 1 = C r^2 with C the minimax constant on |r| <= 2^-12 (-(2pi)^2/2 + 3.2e-6:
// error 3.96e-14, computed with mpmath), so the cosine costs one product.
constexpr int HEAVY_TAB = 2048;
constexpr int HEAVY_TAB_BYTES = HEAVY_TAB * (int)sizeof(double2);
MB_DEV void sincos_rotate(double2 T, double r, double &sn, double &cs) {
    const double u = r * r;
    const double s = r * fma(u, -41.341702240399755, 6.283185307179586);     // sin(2 pi r)
    const double cm1 = u * -19.739205595594533;                            // cos(2 pi r) - 1
    cs = fma(T.x, cm1, fma(-T.y, s, T.x));
    sn = fma(T.y, cm1, fma(T.x, s, T.y));
}

// The heavy tier's shared memory: the staged tile / reduction buffer, then the (cos, sin) table
// (dynamic shared memory: 24 KB + 32 KB is above the 48 KB static limit).
constexpr int HEAVY_DSMEM = FAST_SMEM + HEAVY_TAB_BYTES;

MB_DEV double2 *heavy_table_init(unsigned char *dsm) {
    double2 *tab = reinterpret_cast<double2 *>(dsm + FAST_SMEM);
    for (int i = threadIdx.x; i < HEAVY_TAB; i += FAST_THREADS) {
        double sn, cs;
        sincospi((double)i * (2.0 / HEAVY_TAB), &sn, &cs);
        tab[i] = make_double2(cs, sn);
    }
    return tab;
}

// 1.5 2^35: a sum x in [0, 2^34) units of 2^-32 turn added to it rounds to a multiple of 2^-17
// unit, and the low 51 mantissa bits of the result hold x 2^17.
constexpr double HEAVY_MAGIC = 51539607552.0;

// The heavy term's phase in units of 2^-32 turn, T = L + F mod 2^32 with
//   L = a1 b0 + a0 b1 + d1 gI + psi_hi (+ 2^20)     exact mod 2^32 (IMAD.lo)
//   F = (a0 b0 + a1 c1 + d0 gI + d1 b1) 2^-32       < 2^34, two FP64 chains, one on HEAVY_MAGIC
//     + (a1 c0 + a0 c1 + d1 b0 + d0 b1) 2^-64 + psi_lo   < 5, FP32
// (error <= 2^-16 unit = 2^-48 turn).  The bits of HEAVY_MAGIC + F plus L 2^17 (one 64-bit
// integer multiply-add) are T 2^17: bits [38, 49) are the table index q, bits [0, 38) the offset
// R, and r = R 2^-49 - 2^-12 turn is exact as (2^52 + R) 2^-49 - (8 + 2^-12).
template <int CPT>
MB_DEV void heavy_tile(const ZHeavy *tile, int nt, int zl, int ZL, const CandRegs (&cr)[CPT],
                       double (&acc)[CPT][3], const double2 *tab) {
    for (int jj = zl; jj < nt; jj += ZL) {
        const ZHeavy z = tile[jj];
#pragma unroll
        for (int i = 0; i < CPT; ++i) {
            const uint32_t L = cr[i].a1 * z.b0 + cr[i].a0 * z.b1 + cr[i].d1 * z.gi + z.psi_hi;
            const float low = fmaf(__uint2float_rn(cr[i].a1), z.c0f, fmaf(__uint2float_rn(cr[i].a0), z.c1f,
                              fmaf(__uint2float_rn(cr[i].d1), z.b0f,
                              fmaf(__uint2float_rn(cr[i].d0), z.b1f, z.psi_lo))));
            const double p1 = fma(cr[i].A0, z.b0s, fma(cr[i].A1, z.c1s, (double)low));
            const double p2 = fma(cr[i].D0, z.gis, fma(cr[i].D1, z.b1s, HEAVY_MAGIC));
            const unsigned long long w =
                (unsigned long long)L * 131072ull + (unsigned long long)__double_as_longlong(p1 + p2);
            const uint32_t wh = (uint32_t)(w >> 32);
            const double r = fma(__hiloint2double((int)((wh & 0x3Fu) | 0x43300000u), (int)(uint32_t)w),
                                 1.7763568394002505e-15, -8.000244140625);        // 2^-49, 8 + 2^-12
            double sn, cs;
            sincos_rotate(tab[(wh >> 6) & (HEAVY_TAB - 1)], r, sn, cs);
            acc[i][0] = fma(z.a, cs, acc[i][0]);
            acc[i][1] = fma(z.b, sn, acc[i][1]);
            acc[i][2] = fma(z.d, cs, acc[i][2]);
        }
    }
}

// Stage one zero into a tile record (one thread per zero).  The weight is exp(-k gamma^2), or
// w[j] when the group carries its own weight vector.
MB_DEV void stage_light(const TabView &t, int64_t j, double k, const double *w, ZLight &r) {
    double g = t.gamma[j];
    double a = 2.0 * t.alpha[j] * (w ? w[j] : exp(-k * g * g));
    uint32_t b0 = t.g2[j], b1 = t.g3[j], gi = t.g4[j], c1 = t.g1[j];
    r.b0 = b0; r.b1 = b1; r.gi = gi;
    r.psi32 = (uint32_t)((t.psi[j] + 0x80000000ull) >> 32) + 2u;
    r.b0s = u32_to_f64(b0) * TWO_M32;
    r.c1s = u32_to_f64(c1) * TWO_M32;
    r.gis = u32_to_f64(gi) * TWO_M32;
    r.b1s = u32_to_f64(b1) * TWO_M32;
    r.a = (float)a;
    r.b = (float)(-a * g);
    r.d = (float)(-a * g * g);
    r.pad = 0.f;
}

MB_DEV void stage_light(const TabView &t, int64_t j, double k, const double *w, ZLightF &r) {
    double g = t.gamma[j];
    double a = 2.0 * t.alpha[j] * (w ? w[j] : exp(-k * g * g));
    uint32_t b0 = t.g2[j], b1 = t.g3[j], gi = t.g4[j], c1 = t.g1[j];
    r.b0 = b0; r.b1 = b1;
    // + 1 centres the fused phase's truncation (dropped products in [0, 3) units): error within
    // +-2.4 units of 2^-32 turn
    r.psi32 = (uint32_t)((t.psi[j] + 0x80000000ull) >> 32) + 1u;
    r.b0s = u32_to_f64(b0) * TWO_M32;
    r.c1s = u32_to_f64(c1) * TWO_M32;
    r.gh = fma(u32_to_f64(gi), 4294967296.0, u32_to_f64(b1));
    r.a = (float)a;
    r.b = (float)(-a * g);
    r.d = (float)(-a * g * g);
}

MB_DEV void stage_heavy(const TabView &t, int64_t j, double k, const double *w, ZHeavy &r) {
    double g = t.gamma[j];
    double a = 2.0 * t.alpha[j] * (w ? w[j] : exp(-k * g * g));
    uint32_t c0 = t.g0[j], c1 = t.g1[j], b0 = t.g2[j], b1 = t.g3[j], gi = t.g4[j];
    r.b0 = b0; r.b1 = b1; r.gi = gi;
    r.b0s = u32_to_f64(b0) * TWO_M32;
    r.c1s = u32_to_f64(c1) * TWO_M32;
    r.gis = u32_to_f64(gi) * TWO_M32;
    r.b1s = u32_to_f64(b1) * TWO_M32;
    r.c0f = (float)(u32_to_f64(c0) * TWO_M64);
    r.c1f = (float)(u32_to_f64(c1) * TWO_M64);
    r.b0f = (float)(u32_to_f64(b0) * TWO_M64);
    r.b1f = (float)(u32_to_f64(b1) * TWO_M64);
    const uint64_t ps = t.psi[j];
    r.psi_hi = (uint32_t)(ps >> 32) + (1u << 20);
    r.psi_lo = (float)(u32_to_f64((uint32_t)ps) * TWO_M32);
    r.pad0 = 0.f;
    r.a = a;
    r.b = -a * g;
    r.d = -a * g * g;
}

// Sum res over the nzw warps that share a candidate set, then warp zw==0 writes the partials.
template <int CPT>
MB_DEV void finish_item(const FastItem &it, const FastGroup &gr, double (&res)[CPT][3], int warp, int lane,
                        int zw, int64_t cbase, int64_t cend, double *partial, unsigned char *smem) {
    const int nzw = it.nzw;
    __syncthreads();
    double *red = reinterpret_cast<double *>(smem);
    if (nzw > 1) {
#pragma unroll
        for (int i = 0; i < CPT; ++i)
#pragma unroll
            for (int q = 0; q < 3; ++q) red[((warp * 32 + lane) * CPT + i) * 3 + q] = res[i][q];
        __syncthreads();
        if (zw == 0)
            for (int w2 = 1; w2 < nzw; ++w2)
#pragma unroll
                for (int i = 0; i < CPT; ++i)
#pragma unroll
                    for (int q = 0; q < 3; ++q) res[i][q] += red[(((warp + w2) * 32 + lane) * CPT + i) * 3 + q];
    }
    if (zw == 0) {
#pragma unroll
        for (int i = 0; i < CPT; ++i) {
            int64_t p = cbase + i;
            if (p < cend) {
                double *o = partial + it.pbase + (p - gr.c0) * 3;
                o[0] = res[i][0]; o[1] = res[i][1]; o[2] = res[i][2];
            }
        }
    }
}

template <int CPT, bool FUSED>
MB_DEV void light_item(const FastItem &it, const FastGroup &gr, const TabView &t, const CandView &c,
                       double *partial, unsigned char *smem) {
    using Rec = typename std::conditional<FUSED, ZLightF, ZLight>::type;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nzw = it.nzw;
    const int cgroup = warp / nzw, zw = warp - cgroup * nzw;
    const int64_t cbase = it.c0 + (int64_t)(cgroup * 32 + lane) * CPT;
    const int64_t cend = it.c0 + it.nc;
    CandRegs cr[CPT];
#pragma unroll
    for (int i = 0; i < CPT; ++i) cr[i] = cand_regs(c, cbase + i, cbase + i < cend);
    Rec *tile = reinterpret_cast<Rec *>(smem);
    double res[CPT][3];
#pragma unroll
    for (int i = 0; i < CPT; ++i)
#pragma unroll
        for (int q = 0; q < 3; ++q) res[i][q] = 0.0;
    for (int64_t tb = it.z0; tb < it.z1; tb += LIGHT_TILE) {
        __syncthreads();
        int64_t j = tb + threadIdx.x;
        if (threadIdx.x < LIGHT_TILE && j < it.z1) stage_light(t, j, gr.k, gr.w, tile[threadIdx.x]);
        __syncthreads();
        light_tile<CPT, FUSED>(tile, (int)min((int64_t)LIGHT_TILE, it.z1 - tb), zw, nzw, cr, res);
    }
    finish_item<CPT>(it, gr, res, warp, lane, zw, cbase, cend, partial, smem);
}

template <int CPT>
MB_DEV void heavy_item(const FastItem &it, const FastGroup &gr, const TabView &t, const CandView &c,
                       double *partial, unsigned char *smem, const double2 *tab) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nzw = it.nzw;
    const int cgroup = warp / nzw, zw = warp - cgroup * nzw;
    const int64_t cbase = it.c0 + (int64_t)(cgroup * 32 + lane) * CPT;
    const int64_t cend = it.c0 + it.nc;
    CandRegs cr[CPT];
#pragma unroll
    for (int i = 0; i < CPT; ++i) cr[i] = cand_regs(c, cbase + i, cbase + i < cend);
    ZHeavy *tile = reinterpret_cast<ZHeavy *>(smem);
    double res[CPT][3];
#pragma unroll
    for (int i = 0; i < CPT; ++i) res[i][0] = res[i][1] = res[i][2] = 0.0;
    for (int64_t tb = it.z0; tb < it.z1; tb += HEAVY_TILE) {
        __syncthreads();
        int64_t j = tb + threadIdx.x;
        if (threadIdx.x < HEAVY_TILE && j < it.z1) stage_heavy(t, j, gr.k, gr.w, tile[threadIdx.x]);
        __syncthreads();
        heavy_tile<CPT>(tile, (int)min((int64_t)HEAVY_TILE, it.z1 - tb), zw, nzw, cr, res, tab);
    }
    finish_item<CPT>(it, gr, res, warp, lane, zw, cbase, cend, partial, smem);
}

// Heavy tier: persistent, items pulled from an atomic counter (largest first).  At most 128
// registers per thread: two CTAs per SM.
__global__ void __launch_bounds__(FAST_THREADS, 2)
k2_heavy_kernel(TabView t, CandView c, const FastItem *items, int n_items, const FastGroup *groups,
                int *counter, double *partial) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_item;
    const double2 *s_tab = heavy_table_init(smem);
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int idx = s_item;
        if (idx >= n_items) break;
        const FastItem it = items[idx];
        heavy_item<HEAVY_CPT>(it, groups[it.group], t, c, partial, smem, s_tab);
    }
}

// Light tier: one CTA per item.  MINB sets the register budget (65536 / (256 MINB)).
template <int CPT, int MINB, bool FUSED>
__global__ void __launch_bounds__(FAST_THREADS, MINB)
k2_light_kernel(TabView t, CandView c, const FastItem *items, const FastGroup *groups, double *partial) {
    __shared__ __align__(16) unsigned char smem[FAST_SMEM];
    const FastItem it = items[blockIdx.x];
    light_item<CPT, FUSED>(it, groups[it.group], t, c, partial, smem);
}

// Both tiers in one persistent kernel: two CTAs per SM pull items, so the SMs stay busy to the
// end without a second launch.  The light part runs at the heavy part's register budget
// (launch bounds 256 x 2: at most 128 registers per thread).
//   n_first == 0: one queue, counter[0] over items[0, n_items) (heavy items first or a
//                 cost-ordered list of both tiers);
//   n_first  > 0: paired -- the first CTA to arrive on an SM (counter[2 + smid]) pulls heavy
//                 items [0, n_first) from counter[0], the second light items [n_first, n_items)
//                 from counter[1], so each SM runs one CTA of each tier (FP64 pipe beside XU
//                 pipe); a CTA whose queue is empty takes the other one's.
template <int CPT, bool FUSED>
__global__ void __launch_bounds__(FAST_THREADS, 2)
k2_tiers_kernel(TabView t, CandView c, const FastItem *items, int n_items, int n_first, const FastGroup *groups,
                int *counter, double *partial) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_item, s_queue;
    const double2 *s_tab = heavy_table_init(smem);
    if (threadIdx.x == 0 && n_first > 0) {
        unsigned smid;
        asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
        s_queue = smid < TIERS_COUNTERS - 2 ? atomicAdd(&counter[2 + smid], 1) & 1 : (int)(blockIdx.x & 1);
    }
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            if (n_first == 0) {
                s_item = atomicAdd(counter, 1);
            } else {
                int idx = n_items;
                for (int tries = 0; tries < 2; ++tries) {
                    const int q = s_queue;
                    const int k = atomicAdd(&counter[q], 1);
                    if (q == 0 ? k < n_first : n_first + k < n_items) {
                        idx = q == 0 ? k : n_first + k;
                        break;
                    }
                    s_queue = q ^ 1;
                }
                s_item = idx;
            }
        }
        __syncthreads();
        const int idx = s_item;
        if (idx >= n_items) break;
        const FastItem it = items[idx];
        if (it.tier == 0)
            heavy_item<HEAVY_CPT>(it, groups[it.group], t, c, partial, smem, s_tab);
        else
            light_item<CPT, FUSED>(it, groups[it.group], t, c, partial, smem);
    }
}

// Eight lanes per candidate, four candidates per warp: lane 4r + q sums the chunks r, r + 8, ...
// of candidate 4w + q, so the four lanes of one chunk read 96 consecutive bytes; a fixed shuffle
// tree then adds the eight lanes (deterministic: the order depends only on the chunk count).
constexpr int REDUCE_LANES = 8;
__global__ void fast_reduce_kernel(const FastGroup *groups, int n_groups, const double *partial,
                                   int64_t P, double *val, double *dd, double *dk) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int r = lane >> 2;
    const int64_t p = (t >> 5) * 4 + (lane & 3);
    const bool live = p < P;
    double s0 = 0, s1 = 0, s2 = 0;
    if (live) {
        int lo = 0, hi = n_groups - 1;             // group containing p (groups sorted by c0)
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (groups[mid].c0 <= p) lo = mid;
            else hi = mid - 1;
        }
        const FastGroup gr = groups[lo];
        const int64_t stride = (int64_t)gr.nc * 3;
        const double *o = partial + gr.pbase + (p - gr.c0) * 3 + r * stride;
        int ch = r;
        // four chunks per round, all twelve loads issued before the adds (the rounds are
        // latency-bound otherwise)
        for (; ch + 3 * REDUCE_LANES < gr.n_chunks; ch += 4 * REDUCE_LANES, o += 4 * REDUCE_LANES * stride) {
            double x[4][3];
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int q = 0; q < 3; ++q) x[u][q] = o[u * REDUCE_LANES * stride + q];
            s0 += (x[0][0] + x[1][0]) + (x[2][0] + x[3][0]);
            s1 += (x[0][1] + x[1][1]) + (x[2][1] + x[3][1]);
            s2 += (x[0][2] + x[1][2]) + (x[2][2] + x[3][2]);
        }
        for (; ch < gr.n_chunks; ch += REDUCE_LANES, o += REDUCE_LANES * stride) {
            s0 += o[0]; s1 += o[1]; s2 += o[2];
        }
    }
    for (int off = 16; off >= 4; off >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, off);
        s1 += __shfl_xor_sync(0xffffffffu, s1, off);
        s2 += __shfl_xor_sync(0xffffffffu, s2, off);
    }
    if (live && r == 0) {
        val[p] = s0;
        dd[p] = s1;
        dk[p] = s2;
    }
}
static unsigned reduce_blocks(int64_t P) { return (unsigned)(((P + 3) / 4 * 32 + 255) / 256); }

static int launch_light(const TabView &tv, const FastPlanDev &pd, CandView c, cudaStream_t s) {
    if (pd.n_light == 0) return MB_OK;
    dim3 grid((unsigned)pd.n_light);
    const FastItem *li = pd.items + pd.n_heavy;
    if (pd.fused_phase) {
        switch (pd.light_cpt) {
            case 2: k2_light_kernel<2, 4, true><<<grid, FAST_THREADS, 0, s>>>(tv, c, li, pd.groups, pd.partial); break;
            case 3: k2_light_kernel<3, 3, true><<<grid, FAST_THREADS, 0, s>>>(tv, c, li, pd.groups, pd.partial); break;
            default: k2_light_kernel<4, 2, true><<<grid, FAST_THREADS, 0, s>>>(tv, c, li, pd.groups, pd.partial); break;
        }
    } else {
        switch (pd.light_cpt) {
            case 2: k2_light_kernel<2, 4, false><<<grid, FAST_THREADS, 0, s>>>(tv, c, li, pd.groups, pd.partial); break;
            case 3: k2_light_kernel<3, 3, false><<<grid, FAST_THREADS, 0, s>>>(tv, c, li, pd.groups, pd.partial); break;
            default: k2_light_kernel<4, 2, false><<<grid, FAST_THREADS, 0, s>>>(tv, c, li, pd.groups, pd.partial); break;
        }
    }
    MB_CUDA(cudaGetLastError());
    return MB_OK;
}

// Opt every kernel that holds the heavy table into HEAVY_DSMEM bytes of dynamic shared memory, and
// give every tier kernel the same shared-memory carveout (the largest): an SM switches its L1 /
// shared split only when it is idle, so a light CTA could not take an SM that a heavy CTA (with
// its larger shared-memory need) had just left without one (measured: the two-kernel step
// 1.726 -> 1.689 ms at 4,096 x 466,659 once the carveouts matched).  Once per device and
// context (the attributes belong to the context: after a cudaDeviceReset they are set again).
// Plans call it when they are built, so a first launch inside a stream capture finds it done.
template <typename K>
static int tier_kernel_attributes(K kern, bool heavy_table) {
    if (heavy_table)
        MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, HEAVY_DSMEM));
    MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared));
    return MB_OK;
}

int heavy_smem_attributes() {
    static void *done_ctx[64] = {};             // the context the attributes were set in
    int dev = 0;
    MB_CUDA(cudaGetDevice(&dev));
    void *ctx = current_context();
    if (dev >= 0 && dev < 64 && ctx && done_ctx[dev] == ctx) return MB_OK;
    MB_TRY(tier_kernel_attributes(k2_heavy_kernel, true));
    MB_TRY(tier_kernel_attributes(k2_tiers_kernel<2, true>, true));
    MB_TRY(tier_kernel_attributes(k2_tiers_kernel<3, true>, true));
    MB_TRY(tier_kernel_attributes(k2_tiers_kernel<4, true>, true));
    MB_TRY(tier_kernel_attributes(k2_tiers_kernel<2, false>, true));
    MB_TRY(tier_kernel_attributes(k2_tiers_kernel<3, false>, true));
    MB_TRY(tier_kernel_attributes(k2_tiers_kernel<4, false>, true));
    MB_TRY(tier_kernel_attributes(k2_light_kernel<2, 4, true>, false));
    MB_TRY(tier_kernel_attributes(k2_light_kernel<3, 3, true>, false));
    MB_TRY(tier_kernel_attributes(k2_light_kernel<4, 2, true>, false));
    MB_TRY(tier_kernel_attributes(k2_light_kernel<2, 4, false>, false));
    MB_TRY(tier_kernel_attributes(k2_light_kernel<3, 3, false>, false));
    MB_TRY(tier_kernel_attributes(k2_light_kernel<4, 2, false>, false));
    if (dev >= 0 && dev < 64) done_ctx[dev] = current_context();
    return MB_OK;
}

static int launch_tiers_one(const TabView &tv, const FastPlanDev &pd, CandView c, cudaStream_t s) {
    const unsigned grid = pd.tiers_grid;
    const int n = pd.n_heavy + pd.n_light;
    const int nf = pd.paired ? pd.n_heavy : 0;
    const size_t sm = HEAVY_DSMEM;
#define MB_TIERS(C, F) k2_tiers_kernel<C, F><<<grid, FAST_THREADS, sm, s>>>(tv, c, pd.items_one, n, nf, pd.groups, \
                                                                         pd.counter, pd.partial)
    if (pd.fused_phase) {
        switch (pd.light_cpt) {
            case 2: MB_TIERS(2, true); break;
            case 3: MB_TIERS(3, true); break;
            default: MB_TIERS(4, true); break;
        }
    } else {
        switch (pd.light_cpt) {
            case 2: MB_TIERS(2, false); break;
            case 3: MB_TIERS(3, false); break;
            default: MB_TIERS(4, false); break;
        }
    }
#undef MB_TIERS
    MB_CUDA(cudaGetLastError());
    return MB_OK;
}

// tiers: bit 0 runs the heavy tier, bit 1 the light tier (3 = the full evaluation; a single
// tier is used to time one kernel on its own -- the result then lacks the other tier).  With
// pd.one_kernel and both tiers, k2_tiers_kernel runs every item (its events are the light pair).
int launch_fast(const Table &t, const FastPlanDev &pd, CandView c, double *d_val, double *d_dd,
                double *d_dk, cudaStream_t s, int tiers, const TierEvents *ev) {
    const TabView tv = view(t);
    const bool heavy = (tiers & 1) && pd.n_heavy > 0;
    const bool light = (tiers & 2) && pd.n_light > 0;
    if (heavy || light) MB_TRY(heavy_smem_attributes());
    if (pd.one_kernel && heavy && light) {
        MB_CUDA(cudaMemsetAsync(pd.counter, 0, (pd.paired ? TIERS_COUNTERS : 1) * sizeof(int), s));
        if (ev) MB_CUDA(cudaEventRecord(ev->light0, s));
        MB_TRY(launch_tiers_one(tv, pd, c, s));
        if (ev) MB_CUDA(cudaEventRecord(ev->light1, s));
        fast_reduce_kernel<<<reduce_blocks(c.P), 256, 0, s>>>(pd.groups, pd.n_groups, pd.partial, c.P,
                                                                         d_val, d_dd, d_dk);
        MB_CUDA(cudaGetLastError());
        return MB_OK;
    }
    // with both tiers: fork the heavy tier onto the table's side stream, concurrently with the
    // light tier on s; with one tier everything stays on s
    const bool fork = heavy && light;
    cudaStream_t hs = fork ? t.side : s;
    // a one-tier run: the other tier's partial sums count as zero, not as a previous run's values
    if ((tiers & 3) != 3) MB_CUDA(cudaMemsetAsync(pd.partial, 0, pd.partial_bytes, s));
    if (heavy) {
        if (fork) {
            MB_CUDA(cudaEventRecord(t.ev_fork, s));
            MB_CUDA(cudaStreamWaitEvent(t.side, t.ev_fork, 0));
        }
        MB_CUDA(cudaMemsetAsync(pd.counter, 0, sizeof(int), hs));
        if (ev) MB_CUDA(cudaEventRecord(ev->heavy0, hs));
        k2_heavy_kernel<<<pd.heavy_grid, FAST_THREADS, HEAVY_DSMEM, hs>>>(tv, c, pd.items, pd.n_heavy, pd.groups,
                                                                          pd.counter, pd.partial);
        MB_CUDA(cudaGetLastError());
        if (ev) MB_CUDA(cudaEventRecord(ev->heavy1, hs));
        if (fork) MB_CUDA(cudaEventRecord(t.ev_join, t.side));
    }
    if (light) {
        if (ev) MB_CUDA(cudaEventRecord(ev->light0, s));
        MB_TRY(launch_light(tv, pd, c, s));
        if (ev) MB_CUDA(cudaEventRecord(ev->light1, s));
    }
    if (fork) MB_CUDA(cudaStreamWaitEvent(s, t.ev_join, 0));
    fast_reduce_kernel<<<reduce_blocks(c.P), 256, 0, s>>>(pd.groups, pd.n_groups, pd.partial, c.P,
                                                                     d_val, d_dd, d_dk);
    MB_CUDA(cudaGetLastError());
    return MB_OK;
}

// Issue-rate calibration: independent FFMA chains (full-rate instruction), 8 per thread.
__global__ void __launch_bounds__(256) issue_calibration_kernel(int iters, float *sink) {
    float f[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = 1.0f + 1e-3f * (threadIdx.x + i);
    const float a = 0.99999994f, b = 1e-7f;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) asm volatile("fma.rn.f32 %0, %0, %1, %2;" : "+f"(f[i]) : "f"(a), "f"(b));
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += f[i];
    if (s == 123.25f) sink[0] = s;
}

int calibrate_issue(int device, double *thread_inst_per_s) {
    int sms = 148;
    MB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    float *sink = nullptr;
    MB_CUDA(cudaMalloc(&sink, sizeof(float)));
    cudaEvent_t e0, e1;
    MB_CUDA(cudaEventCreate(&e0));
    MB_CUDA(cudaEventCreate(&e1));
    const int iters = 8192;
    const unsigned grid = (unsigned)sms * 8;
    issue_calibration_kernel<<<grid, 256>>>(64, sink);
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(e0);
        issue_calibration_kernel<<<grid, 256>>>(iters, sink);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        best = std::min(best, ms);
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (e != cudaSuccess) {
        set_error("calibration: %s", cudaGetErrorString(e));
        return MB_ERR_CUDA;
    }
    *thread_inst_per_s = (double)grid * 256 * iters * 8 / (best * 1e-3);
    return MB_OK;
}

// Pipe calibration: eight independent dependency chains per thread of one operation, enough warps
// to fill every scheduler; the rate is thread operations per second.
__global__ void __launch_bounds__(256) mufu_calibration_kernel(int iters, float *sink) {
    float f[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = 0.25f + 1e-3f * (threadIdx.x + i);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; i += 2) {
            asm volatile("sin.approx.f32 %0, %0;" : "+f"(f[i]));
            asm volatile("cos.approx.f32 %0, %0;" : "+f"(f[i + 1]));
        }
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += f[i];
    if (s == 123.25f) sink[0] = s;
}

__global__ void __launch_bounds__(256) dfma_calibration_kernel(int iters, float *sink) {
    double f[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = 1.0 + 1e-3 * (threadIdx.x + i);
    const double a = 0.9999999999, b = 1e-10;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) asm volatile("fma.rn.f64 %0, %0, %1, %2;" : "+d"(f[i]) : "d"(a), "d"(b));
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += f[i];
    if (s == 123.25) sink[0] = (float)s;
}

namespace {
// Best of three timed launches (after one short warm-up) of kern(iters), in thread ops per second
// (8 chains of `iters` operations per thread).
template <typename K>
int time_chains(K kern, unsigned grid, int iters, float *sink, double *rate) {
    cudaEvent_t e0, e1;
    MB_CUDA(cudaEventCreate(&e0));
    MB_CUDA(cudaEventCreate(&e1));
    kern<<<grid, 256>>>(64, sink);
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(e0);
        kern<<<grid, 256>>>(iters, sink);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        best = std::min(best, ms);
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) {
        set_error("calibration: %s", cudaGetErrorString(e));
        return MB_ERR_CUDA;
    }
    *rate = (double)grid * 256 * iters * 8 / (best * 1e-3);
    return MB_OK;
}
}  // namespace

int calibrate_pipes(int device, double *ffma_per_s, double *mufu_per_s, double *dfma_per_s) {
    int sms = 148;
    MB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    float *sink = nullptr;
    MB_CUDA(cudaMalloc(&sink, sizeof(float)));
    const unsigned grid = (unsigned)sms * 8;
    int st = MB_OK;
    if (ffma_per_s) st = time_chains(issue_calibration_kernel, grid, 8192, sink, ffma_per_s);
    if (st == MB_OK && mufu_per_s) st = time_chains(mufu_calibration_kernel, grid, 2048, sink, mufu_per_s);
    if (st == MB_OK && dfma_per_s) st = time_chains(dfma_calibration_kernel, grid, 4096, sink, dfma_per_s);
    cudaFree(sink);
    return st;
}

int heavy_grid_size(int device, unsigned *grid) {
    int sms = 148;
    MB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    // two CTAs per SM (16 warps): the heavy tier is FP64-latency bound with fewer; light CTAs
    // take each SM's registers as the heavy CTAs retire (measured faster than one CTA per SM
    // beside a light CTA)
    *grid = (unsigned)(2 * sms);
    return MB_OK;
}

}  // namespace mb
