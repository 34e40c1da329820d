// Shared device code for the K2 zero-sum kernels (sm_100a).
//
// K2(v,T,k) = 2 sum_{0<gamma<T} exp(-k gamma^2) Re(c e^{i gamma v}),  c = 1/(rho zeta'(rho))
// (reference: certification/certify_K2.py:112-121; search/path1_eval_fast.cpp:41-50).
//
// Fixed-point conventions (host and device):
//   G = gamma/2pi = g_int + g_hi 2^-64 + g_lo 2^-128   (unsigned 64.128)
//   v = v_int + v_frac 2^-64                            (unsigned 64.64)
// In 32-bit limbs: V = v 2^64 = [v3 v2 v1 v0], Gfix = G 2^128 = [g4 g3 g2 g1 g0] with
// g4 = g_int (< 2^32 required), and frac(v G) 2^128 = bits [64,192) of V * Gfix.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "poly_coeffs.h"

#define MB_DEV __device__ __forceinline__

// ---------------------------------------------------------------- candidates

// A candidate with its FP64 offset delta folded into the 64.64 fixed point
// (v' = v + delta rounded to the nearest 2^-64).  Requires |delta| < 2^62.
struct Cand64 {
    uint64_t vi, vf;
};

// The fold proper, kept out of line: it runs once per candidate before a kernel's zero loop, and
// inlined it took two more registers from (and reshuffled) the light tier's loop, which ran 5%
// slower (1.355 against 1.289 ms for the light tier alone at 4,096 x 466,659).
static __device__ __noinline__ Cand64 fold_delta_nonzero(uint64_t vi, uint64_t vf, double delta) {
    Cand64 c{vi, vf};
    {
        // delta = M 2^(e - 53) exactly (|M| < 2^53), so delta 2^64 = M 2^sh: its 128-bit magnitude,
        // rounded to the nearest integer (half up) when sh < 0, is added to or subtracted from v.
        // Every step is exact (1 + delta, say, would round for small negative delta).
        int e;
        const double m = frexp(delta, &e);
        const uint64_t am = (uint64_t)fabs(ldexp(m, 53));
        const int sh = e + 11;                          // e - 53 + 64
        uint64_t hi = 0, lo = 0;
        if (sh >= 64) {
            hi = am << (sh - 64);
        } else if (sh > 0) {
            hi = am >> (64 - sh);
            lo = am << sh;
        } else if (sh == 0) {
            lo = am;
        } else if (sh > -64) {
            lo = (am + (1ull << (-sh - 1))) >> (-sh);
        }
        if (delta > 0.0) {
            const uint64_t nf = vf + lo;
            c.vf = nf;
            c.vi = vi + hi + (nf < vf ? 1u : 0u);
        } else {
            c.vf = vf - lo;
            c.vi = vi - hi - (vf < lo ? 1u : 0u);
        }
    }
    return c;
}

MB_DEV Cand64 fold_delta(uint64_t vi, uint64_t vf, double delta) {
    if (delta == 0.0) return Cand64{vi, vf};
    return fold_delta_nonzero(vi, vf, delta);
}

// ---------------------------------------------------------------- exact phase

// floor(frac(v G) 2^128) as (hi, lo) -- exact, integer pipe only.
// Product scanning over 32-bit limbs with carry chains: column k of V*Gfix takes lo(v_i g_j)
// for i+j=k and hi(v_i g_j) for i+j=k-1; columns 0..5 are formed (columns >= 6 are integer
// multiples of 1 after the 2^-192 scaling and are dropped).
MB_DEV void phase128_exact(uint32_t v0, uint32_t v1, uint32_t v2, uint32_t v3, uint32_t g0,
                           uint32_t g1, uint32_t g2, uint32_t g3, uint32_t g4, uint64_t &hi,
                           uint64_t &lo) {
    // tA, tB, tC: 96-bit rotating column accumulator (PTX registers)
    uint32_t r2, r3, r4, r5;
    // column 0: lo(v0 g0); we only need its carry-producing high part into column 1
    asm("{\n\t"
        ".reg .u32 c0, tA, tB, tC;\n\t"
        // col 0
        "mul.lo.u32 c0, %4, %8;\n\t"
        "mul.hi.u32 tA, %4, %8;\n\t"        // t0 = hi(v0 g0) -> col 1
        "mov.u32 tB, 0;\n\t"
        "mov.u32 tC, 0;\n\t"
        // col 1: lo(v0 g1) + lo(v1 g0) + t0 ; hi(..) -> col 2
        "mad.lo.cc.u32 tA, %4, %9, tA;\n\t"
        "madc.hi.cc.u32 tB, %4, %9, tB;\n\t"
        "addc.u32 tC, tC, 0;\n\t"
        "mad.lo.cc.u32 tA, %5, %8, tA;\n\t"
        "madc.hi.cc.u32 tB, %5, %8, tB;\n\t"
        "addc.u32 tC, tC, 0;\n\t"
        // shift: col1 result dropped (below 2^64), carry into col 2
        // col 2
        "mad.lo.cc.u32 tB, %4, %10, tB;\n\t"
        "madc.hi.cc.u32 tC, %4, %10, tC;\n\t"
        "addc.u32 tA, 0, 0;\n\t"
        "mad.lo.cc.u32 tB, %5, %9, tB;\n\t"
        "madc.hi.cc.u32 tC, %5, %9, tC;\n\t"
        "addc.u32 tA, tA, 0;\n\t"
        "mad.lo.cc.u32 tB, %6, %8, tB;\n\t"
        "madc.hi.cc.u32 tC, %6, %8, tC;\n\t"
        "addc.u32 tA, tA, 0;\n\t"
        "mov.u32 %0, tB;\n\t"                 // r2
        // col 3 (accumulator now t=(tC,tA,new))
        "mad.lo.cc.u32 tC, %4, %11, tC;\n\t"
        "madc.hi.cc.u32 tA, %4, %11, tA;\n\t"
        "addc.u32 tB, 0, 0;\n\t"
        "mad.lo.cc.u32 tC, %5, %10, tC;\n\t"
        "madc.hi.cc.u32 tA, %5, %10, tA;\n\t"
        "addc.u32 tB, tB, 0;\n\t"
        "mad.lo.cc.u32 tC, %6, %9, tC;\n\t"
        "madc.hi.cc.u32 tA, %6, %9, tA;\n\t"
        "addc.u32 tB, tB, 0;\n\t"
        "mad.lo.cc.u32 tC, %7, %8, tC;\n\t"
        "madc.hi.cc.u32 tA, %7, %8, tA;\n\t"
        "addc.u32 tB, tB, 0;\n\t"
        "mov.u32 %1, tC;\n\t"                 // r3
        // col 4 (t=(tA,tB,new))
        "mad.lo.cc.u32 tA, %4, %12, tA;\n\t"
        "madc.hi.cc.u32 tB, %4, %12, tB;\n\t"
        "mad.lo.cc.u32 tA, %5, %11, tA;\n\t"
        "madc.hi.cc.u32 tB, %5, %11, tB;\n\t"
        "mad.lo.cc.u32 tA, %6, %10, tA;\n\t"
        "madc.hi.cc.u32 tB, %6, %10, tB;\n\t"
        "mad.lo.cc.u32 tA, %7, %9, tA;\n\t"
        "madc.hi.u32 tB, %7, %9, tB;\n\t"
        "mov.u32 %2, tA;\n\t"                 // r4
        // col 5: lo products only (their highs are >= 2^192)
        "mad.lo.u32 tB, %5, %12, tB;\n\t"
        "mad.lo.u32 tB, %6, %11, tB;\n\t"
        "mad.lo.u32 tB, %7, %10, tB;\n\t"
        "mov.u32 %3, tB;\n\t"                 // r5
        "}"
        : "=r"(r2), "=r"(r3), "=r"(r4), "=r"(r5)
        : "r"(v0), "r"(v1), "r"(v2), "r"(v3), "r"(g0), "r"(g1), "r"(g2), "r"(g3), "r"(g4));
    hi = ((uint64_t)r5 << 32) | r4;
    lo = ((uint64_t)r3 << 32) | r2;
}

// ---------------------------------------------------------------- exact small conversions

// Exact double of a 32-bit unsigned integer without the conversion unit
// (2^52 + x has x in its low mantissa bits).
MB_DEV double u32_to_f64(uint32_t x) {
    return __hiloint2double(0x43300000, (int)x) - 4503599627370496.0;
}
// Exact double of a signed 32-bit integer.
MB_DEV double s32_to_f64(int32_t x) {
    return __hiloint2double(0x43300000, (int)((uint32_t)x ^ 0x80000000u)) - 4503601774854144.0;
}
// Signed 64-bit word interpreted as turns in [-1/2, 1/2): x 2^-64, rounded to double.
MB_DEV double s64_turns_to_f64(uint64_t w) {
    double h = s32_to_f64((int32_t)(uint32_t)(w >> 32));
    double l = u32_to_f64((uint32_t)w);
    return fma(h, 2.3283064365386963e-10, l * 5.421010862427522e-20);
}

// ---------------------------------------------------------------- trig in turns

// sin(2 pi t), cos(2 pi t) for |t| <= 1/2 (FP64), by the half-angle pair
// s = sin(pi t), c = cos(pi t): sin(2 pi t) = 2 s c, cos(2 pi t) = 1 - 2 s^2.
// No quadrant selection, so no integer work; ~21 FP64 operations.
MB_DEV void sincos_turns_half(double t, double &s2, double &c2) {
    double u = t * t;
    double ps = HALF_S[8];
#pragma unroll
    for (int i = 7; i >= 0; --i) ps = fma(ps, u, HALF_S[i]);
    double pc = HALF_C[9];
#pragma unroll
    for (int i = 8; i >= 0; --i) pc = fma(pc, u, HALF_C[i]);
    double s = t * ps;
    s2 = 2.0 * s * pc;
    c2 = fma(-2.0 * s, s, 1.0);
}

// 1.5 2^52: adding it rounds a double of magnitude < 2^51 to an integer held in the low
// mantissa word.
constexpr double MB_MAGIC = 6755399441055744.0;

// sin/cos(2 pi y) for any y (turns) via quarter-turn reduction; FP64, error ~6e-14
// (the degree-5 QUAD polynomials on |r| <= 1/8).
MB_DEV void sincos_turns_quad(double y, double &sn, double &cs) {
    double m = fma(y, 4.0, MB_MAGIC);
    int q = __double2loint(m);
    double r = fma(-0.25, m - MB_MAGIC, y);          // |r| <= 1/8 (exact)
    double u = r * r;
    double ps = QUAD_S[5];
#pragma unroll
    for (int k = 4; k >= 0; --k) ps = fma(ps, u, QUAD_S[k]);
    double pc = QUAD_C[5];
#pragma unroll
    for (int k = 4; k >= 0; --k) pc = fma(pc, u, QUAD_C[k]);
    double s = r * ps;
    // rotate by q quarter turns: q=0 (s,c) 1 (c,-s) 2 (-s,-c) 3 (-c,s)
    double S = (q & 1) ? pc : s;
    double Cc = (q & 1) ? s : pc;
    int sgn_s = (q & 2) << 30;
    int sgn_c = ((q ^ (q >> 1)) & 1) << 31;
    sn = __hiloint2double(__double2hiint(S) ^ sgn_s, __double2loint(S));
    cs = __hiloint2double(__double2hiint(Cc) ^ sgn_c, __double2loint(Cc));
}

// ---------------------------------------------------------------- reductions

MB_DEV double warp_sum_xor(double x, int width) {
    for (int o = width >> 1; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}
