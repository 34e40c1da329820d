// The 32-bit light-tier phase shared by the chosen form (k2_fast.cu) and the leaf screen
// (k2_screen.cu).
//
// With v = a1 2^32 + a0 + d1 2^-32 + d0 2^-64 and G = gI + b1 2^-32 + b0 2^-64 + c1 2^-96 + ...
// (32-bit limbs):
//   frac(vG) 2^32 = [a1 b0 + a0 b1 + d1 gI]                   (exact mod 2^32, three IMAD.lo)
//                 + (a0 b0 + a1 c1 + d0 gI + d1 b1) 2^-32       (< 2^34, four DFMA on top of
//                                                               1.5 2^52, so the low mantissa
//                                                               word holds the rounded sum)
// and the dropped products are below 4 units of 2^-32 turn.
#pragma once
#include "k2_common.cuh"
#include "k2_internal.h"

namespace mb {

constexpr double MAGIC = 6755399441055744.0;   // 1.5 2^52
constexpr double TWO_M32 = 2.3283064365386963e-10;
constexpr double TWO_M64 = 5.421010862427522e-20;
constexpr double TWO_M96 = 1.2621774483536189e-29;

// Candidate registers of the light and heavy phases.
struct CandRegs {
    uint32_t a0, a1, d1, d0;
    double A0, A1, D0, D1;      // exact doubles of the limbs a0, a1, d0, d1
    double VF;                  // v_frac 2^-64 rounded to double (light_phase32_fused)
};

MB_DEV CandRegs cand_regs_of(Cand64 v) {
    CandRegs r;
    r.a0 = (uint32_t)v.vi;
    r.a1 = (uint32_t)(v.vi >> 32);
    r.d1 = (uint32_t)(v.vf >> 32);
    r.d0 = (uint32_t)v.vf;
    r.A0 = u32_to_f64(r.a0);
    r.A1 = u32_to_f64(r.a1);
    r.D0 = u32_to_f64((uint32_t)v.vf);
    r.D1 = u32_to_f64(r.d1);
    r.VF = __ull2double_rn(v.vf) * TWO_M64;
    return r;
}

MB_DEV CandRegs cand_regs(const CandView &c, int64_t p, bool valid) {
    Cand64 v{0, 0};
    if (valid) v = fold_delta(c.vi[p], c.vf[p], c.delta ? c.delta[p] : 0.0);
    return cand_regs_of(v);
}

// add + frac(vG) 2^32 mod 2^32 to within a few units; the zero's limbs b0, b1, gI and its
// scaled doubles b0s = b0 2^-32, c1s = c1 2^-32, gis = gI 2^-32, b1s = b1 2^-32.  The four
// middle products form two independent DFMA chains (each rounded to an integer on top of
// 1.5 2^52; four roundings of <= 1/2 unit in all), so the dependent latency is two DFMAs.
MB_DEV uint32_t light_phase32(const CandRegs &c, uint32_t b0, uint32_t b1, uint32_t gi, double b0s, double c1s,
                              double gis, double b1s, uint32_t add) {
    const uint32_t lo32 = c.a1 * b0 + c.a0 * b1 + c.d1 * gi + add;
    const double R1 = fma(c.A0, b0s, fma(c.A1, c1s, MAGIC));
    const double R2 = fma(c.D0, gis, fma(c.D1, b1s, MAGIC));
    return lo32 + (uint32_t)__double2loint(R1) + (uint32_t)__double2loint(R2);
}

// The same phase when G's integer part gI is below 2^19 (gamma < 3.29e6): the whole fraction part
// of v enters through one product,
//   v_frac 2^-64 (gI + b1 2^-32) 2^32 = VF gh,   gh = gI 2^32 + b1 (exact, < 2^51),
// rounded to an integer on top of 1.5 2^52 (VF carries v_frac to 53 bits: <= 2^-3 unit of error),
// so d1 gI leaves the integer sum and d0 gI, d1 b1 leave the FP64 one: 2 IMAD.lo + 3 DFMA.
// Dropped: a1 c0 2^-64, a0 c1 2^-64 and v_frac b0 2^-96, below 3 units in all.
MB_DEV uint32_t light_phase32_fused(const CandRegs &c, uint32_t b0, uint32_t b1, double b0s, double c1s, double gh,
                                    uint32_t add) {
    const uint32_t lo32 = c.a1 * b0 + c.a0 * b1 + add;
    const double R1 = fma(c.A0, b0s, fma(c.A1, c1s, MAGIC));
    const double R2 = fma(c.VF, gh, MAGIC);
    return lo32 + (uint32_t)__double2loint(R1) + (uint32_t)__double2loint(R2);
}

}  // namespace mb
