/*
 * CPU oracle for the K2 zero sum -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load this
 * library, and only as the checker.  The product path (mertens_bound_b200) never calls it.
 *
 * What it restates (reference = bzyzz/mertens_bound):
 *   K2(v,T,k) = 2 sum_{0<gamma<T} exp(-k gamma^2) Re(c e^{i gamma v}),  c = 1/(rho zeta'(rho))
 *     -- certification/certify_K2.py:112-121 (term = 2 w Re(c exp(i g v))), THEOREM.md:7.
 *   The phase gamma v / 2pi mod 1 reduced exactly in integers
 *     -- search/path1_eval_fast.cpp:41-46 (u128 fixed-point product, top 64 bits kept),
 *        legacy/superseded/certify_peak2_600k.py:181-187 (same product in Python ints).
 *   compute_peak_AB / polish_peaks_with_weights semantics
 *     -- search/path1_eval_fast.cpp:15-53 and :58-143 (restated in orc_ref_peak_AB /
 *        orc_ref_polish below, line for line in meaning, single-threaded).
 *   The enumerators' CPU leaf screen ZeroData::fast_screen
 *     -- search/fast_mertens_enum.cpp:99-104 (16384-entry FP32 cosine table, offset steps) and
 *        :108-142 (two stages of 64 zeros, 7 offsets, thresholds 0.810 / 0.875), restated in
 *        orc_fast_screen below, OpenMP over leaves as the enumerator runs it.
 *
 * Fixed-point conventions used throughout this repository:
 *   G = gamma/2pi as unsigned 64.128 fixed point: G = g_int + g_hi 2^-64 + g_lo 2^-128
 *       (three u64 limbs per zero, stored [g_int, g_hi, g_lo]).
 *   v = v_int + v_frac 2^-64 (unsigned 64.64), plus an optional FP64 offset delta.
 *   phase128(v, G) = floor(frac(v G) 2^128), returned as (hi, lo) u64 words.
 *
 * Arithmetic: exact unsigned __int128 for the phase, IEEE binary128 (__float128,
 * libquadmath) for cos/sin/exp and the sums, so the oracle's own rounding error is
 * ~1e-30 relative -- far below the 1e-10 parity bar.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <quadmath.h>

typedef unsigned __int128 u128;

#define Q_2PI (2.0Q * M_PIq)

/* floor(frac(v G) * 2^128) for v = vi + vf 2^-64 and G = gi + g1 2^-64 + g2 2^-128.
 * V = vi 2^64 + vf and Gfix = gi 2^128 + g1 2^64 + g2 are integers; the wanted bits are
 * bits [64, 192) of V * Gfix.  Partial products below bit 64 can only carry through the
 * word at bits [64,128), which is summed exactly here. */
static inline void phase128(uint64_t vi, uint64_t vf, uint64_t gi, uint64_t g1, uint64_t g2,
                            uint64_t *hi, uint64_t *lo) {
    u128 t0 = (u128)vf * g2;          /* at 2^0   */
    u128 t1 = (u128)vf * g1;          /* at 2^64  */
    u128 t2 = (u128)vi * g2;          /* at 2^64  */
    u128 t3 = (u128)vf * gi;          /* at 2^128 */
    u128 t4 = (u128)vi * g1;          /* at 2^128 */
    u128 w1 = (u128)(uint64_t)(t0 >> 64) + (uint64_t)t1 + (uint64_t)t2;
    uint64_t w2 = (uint64_t)(t1 >> 64) + (uint64_t)(t2 >> 64) + (uint64_t)t3 + (uint64_t)t4 +
                  (uint64_t)(w1 >> 64);
    *hi = w2;
    *lo = (uint64_t)w1;
}

void orc_phase128(int64_t P, const uint64_t *v_int, const uint64_t *v_frac, int64_t N,
                  const uint64_t *G3, uint64_t *out_hi, uint64_t *out_lo) {
    for (int64_t p = 0; p < P; ++p)
        for (int64_t j = 0; j < N; ++j)
            phase128(v_int[p], v_frac[p], G3[3 * j], G3[3 * j + 1], G3[3 * j + 2],
                     &out_hi[p * N + j], &out_lo[p * N + j]);
}

static inline __float128 G_quad(const uint64_t *g) {
    return (__float128)g[0] + ldexpq((__float128)g[1], -64) + ldexpq((__float128)g[2], -128);
}

/* K2 value and its two derivatives, in binary128.
 *   val = 2 sum w Re(c e^{i th}),  dd = dK2/ddelta = -2 sum w gam Im(c e^{i th}),
 *   dk  = dK2/dk = -2 sum w gam^2 Re(c e^{i th}),  th = 2pi frac(v G) + gam delta,
 *   w = exp(-k gam^2) (or wts[j] when wts is given: the search drivers' other weight
 *   kernels, search/eval_tech1_600k.py:243-249), gam = 2pi G (exact G, not the FP64 gamma).
 * Zeros j < n_use are summed (the caller applies the cutoff gamma < T).
 * gam and w depend on the zero only, so they are formed once per zero (in binary128, the same
 * operations as per term) and shared by every candidate.
 * Each output is returned as a double pair (hi, lo) with hi + lo = the binary128 sum
 * rounded to ~106 bits, so tests can see errors far below one FP64 ulp. */
void orc_k2_quad_w(int64_t P, const uint64_t *v_int, const uint64_t *v_frac, const double *delta,
                   int64_t n_use, const uint64_t *G3, const double *c_re, const double *c_im,
                   double k, const double *wts, double *out /* P x 6: val hi,lo, dd hi,lo, dk hi,lo */) {
    __float128 *gq = (__float128 *)malloc(sizeof(__float128) * (size_t)(n_use > 0 ? n_use : 1));
    __float128 *wq = (__float128 *)malloc(sizeof(__float128) * (size_t)(n_use > 0 ? n_use : 1));
    if (!gq || !wq) {
        free(gq);
        free(wq);
        for (int64_t i = 0; i < 6 * P; ++i) out[i] = NAN;
        return;
    }
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < n_use; ++j) {
        gq[j] = Q_2PI * G_quad(&G3[3 * j]);
        wq[j] = wts ? (__float128)wts[j] : expq(-(__float128)k * gq[j] * gq[j]);
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t p = 0; p < P; ++p) {
        __float128 sv = 0, sd = 0, sk = 0;
        __float128 dq = delta ? (__float128)delta[p] : 0;
        for (int64_t j = 0; j < n_use; ++j) {
            uint64_t hi, lo;
            phase128(v_int[p], v_frac[p], G3[3 * j], G3[3 * j + 1], G3[3 * j + 2], &hi, &lo);
            const __float128 gam = gq[j], w = wq[j];
            __float128 fr = ldexpq((__float128)hi, -64) + ldexpq((__float128)lo, -128);
            __float128 th = Q_2PI * fr + gam * dq;
            __float128 s, c;
            sincosq(th, &s, &c);
            __float128 re = (__float128)c_re[j] * c - (__float128)c_im[j] * s;
            __float128 im = (__float128)c_re[j] * s + (__float128)c_im[j] * c;
            sv += w * re;
            sd += w * gam * im;
            sk += w * gam * gam * re;
        }
        __float128 r[3] = {2 * sv, -2 * sd, -2 * sk};
        for (int i = 0; i < 3; ++i) {
            double h = (double)r[i];
            out[6 * p + 2 * i] = h;
            out[6 * p + 2 * i + 1] = (double)(r[i] - (__float128)h);
        }
    }
    free(gq);
    free(wq);
}

void orc_k2_quad(int64_t P, const uint64_t *v_int, const uint64_t *v_frac, const double *delta,
                 int64_t n_use, const uint64_t *G3, const double *c_re, const double *c_im,
                 double k, double *out) {
    orc_k2_quad_w(P, v_int, v_frac, delta, n_use, G3, c_re, c_im, k, NULL, out);
}

/* A_j = 2 Re(c_j e^{i th}), B_j = 2 Im(c_j e^{i th}) at th = 2pi frac(v G_j) + gam_j delta, in
 * binary128 rounded to FP64: the restatement of compute_exact_mpfr_AB
 * (search/path1_kernel_opt.py:71-91), with the exact integer phase standing in for the 256-bit
 * mpfr product.  Output row-major (P, n_use). */
void orc_exact_AB(int64_t P, const uint64_t *v_int, const uint64_t *v_frac, const double *delta,
                  int64_t n_use, const uint64_t *G3, const double *c_re, const double *c_im, double *A,
                  double *B) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t p = 0; p < P; ++p) {
        __float128 dq = delta ? (__float128)delta[p] : 0;
        for (int64_t j = 0; j < n_use; ++j) {
            uint64_t hi, lo;
            phase128(v_int[p], v_frac[p], G3[3 * j], G3[3 * j + 1], G3[3 * j + 2], &hi, &lo);
            __float128 gam = Q_2PI * G_quad(&G3[3 * j]);
            __float128 fr = ldexpq((__float128)hi, -64) + ldexpq((__float128)lo, -128);
            __float128 s, c;
            sincosq(Q_2PI * fr + gam * dq, &s, &c);
            A[p * n_use + j] = (double)(2 * ((__float128)c_re[j] * c - (__float128)c_im[j] * s));
            B[p * n_use + j] = (double)(2 * ((__float128)c_re[j] * s + (__float128)c_im[j] * c));
        }
    }
}

/* Absolute-value sum 2 sum w |c| over the first n_use zeros (binary128), the quantity
 * certify_K2.py:119 accumulates as absS. */
double orc_abs_sum(int64_t n_use, const uint64_t *G3, const double *c_re, const double *c_im, double k) {
    __float128 s = 0;
    for (int64_t j = 0; j < n_use; ++j) {
        __float128 gam = Q_2PI * G_quad(&G3[3 * j]);
        __float128 w = expq(-(__float128)k * gam * gam);
        s += 2 * w * hypotq((__float128)c_re[j], (__float128)c_im[j]);
    }
    return (double)s;
}

/* gamma rounded to the nearest double from exact G (binary128 product, then one
 * rounding; correct except for ties closer than 2^-60 ulp). */
void orc_gamma_from_G(int64_t N, const uint64_t *G3, double *gamma) {
    for (int64_t j = 0; j < N; ++j) gamma[j] = (double)(Q_2PI * G_quad(&G3[3 * j]));
}

/* ---- restatement of the reference's C-ABI evaluator (search/path1_eval_fast.cpp) ---- */

/* path1_eval_fast.cpp:15-53: x = y 2^30 as u128; xh = x >> 48, xl = x mod 2^48;
 * ph = xh ghi + xl glo - psi (mod 2^128); th = top64 * 2pi/2^64 + gamma dy0;
 * A = 2 alpha cos th, B = 2 alpha sin th.  Single-threaded restatement. */
void orc_ref_peak_AB(int n_peaks, const uint64_t *x_lo, const uint64_t *x_hi, const double *dy0,
                     int n_zeros, const double *alpha, const double *gamma, const uint64_t *ghi_lo,
                     const uint64_t *ghi_hi, const uint64_t *glo_lo, const uint64_t *glo_hi,
                     const uint64_t *psi_lo, const uint64_t *psi_hi, double *out_A, double *out_B,
                     uint64_t *out_top /* optional: n_peaks x n_zeros top64 words */) {
    const double scale = 2.0 * M_PI * ldexp(1.0, -64);
    for (int p = 0; p < n_peaks; ++p) {
        u128 x = ((u128)x_hi[p] << 64) | x_lo[p];
        uint64_t xh = (uint64_t)(x >> 48);
        uint64_t xl = (uint64_t)(x & (((u128)1 << 48) - 1));
        for (int i = 0; i < n_zeros; ++i) {
            u128 ghi = ((u128)ghi_hi[i] << 64) | ghi_lo[i];
            u128 glo = ((u128)glo_hi[i] << 64) | glo_lo[i];
            u128 psi = ((u128)psi_hi[i] << 64) | psi_lo[i];
            u128 ph = (u128)xh * ghi + (u128)xl * glo - psi;
            uint64_t top = (uint64_t)(ph >> 64);
            if (out_top) out_top[(size_t)p * n_zeros + i] = top;
            double th = (double)top * scale + gamma[i] * dy0[p];
            if (out_A) out_A[(size_t)p * n_zeros + i] = 2.0 * alpha[i] * cos(th);
            if (out_B) out_B[(size_t)p * n_zeros + i] = 2.0 * alpha[i] * sin(th);
        }
    }
}

/* path1_eval_fast.cpp:58-143: per peak h0 = sum w A; optional grid of 2 steps + 1 shifts
 * over the first min(n, 4096) zeros; up to 6 Newton steps on ddy (step clamped to
 * +-1e-4, stop when |step| < 1e-13 or |f''| <= 1e-12); keep the larger |h|. */
void orc_ref_polish(int n_peaks, int n_zeros, const double *A, const double *B, const double *gamma,
                    const double *w, double grid_half_width, int grid_steps, double *out_h_unpol,
                    double *out_h_pol, double *out_ddy_pol) {
    for (int p = 0; p < n_peaks; ++p) {
        const double *Ap = A + (size_t)p * n_zeros, *Bp = B + (size_t)p * n_zeros;
        double h0 = 0.0;
        for (int i = 0; i < n_zeros; ++i) h0 += w[i] * Ap[i];
        out_h_unpol[p] = h0;
        double best_ddy = 0.0, best_abs = fabs(h0);
        int k_scan = n_zeros < 4096 ? n_zeros : 4096;
        if (grid_steps > 0) {
            for (int m = -grid_steps; m <= grid_steps; ++m) {
                double ddy = (grid_half_width * m) / grid_steps, hs = 0.0;
                for (int i = 0; i < k_scan; ++i) {
                    double th = gamma[i] * ddy;
                    hs += w[i] * (Ap[i] * cos(th) - Bp[i] * sin(th));
                }
                if (fabs(hs) > best_abs) { best_abs = fabs(hs); best_ddy = ddy; }
            }
        }
        double ddy = best_ddy;
        for (int it = 0; it < 6; ++it) {
            double f = 0, fp = 0, fpp = 0;
            for (int i = 0; i < n_zeros; ++i) {
                double g = gamma[i], th = g * ddy, c = cos(th), s = sin(th);
                double val = Ap[i] * c - Bp[i] * s;
                double dval = g * (-Ap[i] * s - Bp[i] * c);
                f += w[i] * val; fp += w[i] * dval; fpp += w[i] * (-g * g * val);
            }
            (void)f;
            if (fabs(fpp) > 1e-12) {
                double step = fp / fpp;
                if (step > 1e-4) step = 1e-4;
                if (step < -1e-4) step = -1e-4;
                ddy -= step;
                if (fabs(step) < 1e-13) break;
            } else {
                break;
            }
        }
        double hf = 0.0;
        for (int i = 0; i < n_zeros; ++i) {
            double th = gamma[i] * ddy;
            hf += w[i] * (Ap[i] * cos(th) - Bp[i] * sin(th));
        }
        if (fabs(h0) > fabs(hf)) { out_h_pol[p] = h0; out_ddy_pol[p] = 0.0; }
        else { out_h_pol[p] = hf; out_ddy_pol[p] = ddy; }
    }
}

/* ZeroData::fast_screen over P leaves x (u128, the enumerators' x = floor(y 2^30)) on the
 * reference's table layout; pass[p] = 1 when the leaf survives both stages.  Returns the number of
 * passing leaves.  The cosine table and step indices are built per call as the reference builds
 * them once per table (search/fast_mertens_enum.cpp:99-104; offset step 0.0014). */
int64_t orc_fast_screen(int64_t P, const uint64_t *x_lo, const uint64_t *x_hi, const uint64_t *ghi_lo,
                        const uint64_t *ghi_hi, const uint64_t *glo_lo, const uint64_t *glo_hi,
                        const uint64_t *psi_lo, const uint64_t *psi_hi, const double *two_astar,
                        const double *gamma, uint8_t *pass) {
    static float lut[16384];
    uint32_t st[128];
    for (int k = 0; k < 16384; ++k) lut[k] = (float)cos(2.0 * M_PI * (double)k / 16384.0);
    for (int i = 0; i < 128; ++i)
        st[i] = ((uint32_t)llround(gamma[i] * 0.0014 * (16384.0 / (2.0 * M_PI)))) & 16383u;
    int64_t n_pass = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : n_pass)
    for (int64_t p = 0; p < P; ++p) {
        const u128 x = ((u128)x_hi[p] << 64) | x_lo[p];
        const uint64_t xh = (uint64_t)(x >> 48);
        const uint64_t xl = (uint64_t)(x & (((u128)1 << 48) - 1));
        float s[7] = {0, 0, 0, 0, 0, 0, 0};
        int ok = 1;
        for (int stage = 0; stage < 2 && ok; ++stage) {
            for (int i = 64 * stage; i < 64 * stage + 64; ++i) {
                const u128 ghi = ((u128)ghi_hi[i] << 64) | ghi_lo[i];
                const u128 glo = ((u128)glo_hi[i] << 64) | glo_lo[i];
                const u128 psi = ((u128)psi_hi[i] << 64) | psi_lo[i];
                const u128 ph = (u128)xh * ghi + (u128)xl * glo - psi;
                const uint32_t i0 = (uint32_t)((uint64_t)(ph >> 64) >> 50);
                const float w = (float)two_astar[i];
                for (int m = -3; m <= 3; ++m) s[m + 3] += w * lut[(i0 + (uint32_t)m * st[i]) & 16383u];
            }
            float mx = 0.f;
            for (int m = 0; m < 7; ++m) mx = fmaxf(mx, fabsf(s[m]));
            ok = mx >= (stage == 0 ? 0.810f : 0.875f);
        }
        pass[p] = (uint8_t)ok;
        n_pass += ok;
    }
    return n_pass;
}
