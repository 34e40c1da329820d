// Certified interval evaluation of K2 with directed rounding.
//
// Returns [lo, hi] containing the exact value of
//   K2 = 2 sum_{gamma_j < T} exp(-k gamma_j^2) Re(c_j e^{i gamma_j v})
// for the table's exact G_j = gamma_j/2pi (64.128), exact FP64 c_j, gamma_j = 2pi G_j (the FP64
// gamma is within 4 ulp of it, checked at table creation), exact k, and v = v_int + v_frac 2^-64
// widened by an optional radius v_rad.  Term by term (certification/certify_K2.py:116-121
// does the same sum in Arb balls):
//   phase    floor(frac(v G) 2^128), exact; quadrant q from its top two bits; the rest
//            r in [m 2^-62, (m+1) 2^-62] (directed conversions); r > 1/2 uses 1 - r with
//            sine and cosine exchanged, so x = (pi/2) r lies in [0, pi/4 + 2^-60].
//   sin, cos Taylor polynomials of sin x / x (9 terms) and cos x (10 terms) in u = x^2,
//            coefficients as outward-rounded intervals, Horner with __fma_rd / __fma_ru, plus
//            the Lagrange remainders x^19/19! and x^20/20!.
//   weight   w in [exp(-k gamma_hi^2)(1 - 2^-51), exp(-k gamma_lo^2)(1 + 2^-51)]: CUDA's exp()
//            has a documented maximum error of 1 ulp; the bound allows 2.
//   term     2 w (Re c cos - Im c sin) in interval arithmetic, widened by
//            2 w_hi (|c| gamma_hi v_rad + term_rad_j).
//   sums     per thread, then warp / block / chunk reductions, lower ends with __dadd_rd and
//            upper ends with __dadd_ru.  Also an upper bound of sum 2 w |c| (certify_K2's absS).
#include <algorithm>
#include <cmath>

#include "k2_common.cuh"
#include "k2_internal.h"

namespace mb {

struct Ival {
    double lo, hi;
};

MB_DEV Ival horner_step(const Ival &u, const Ival &p, double clo, double chi) {
    // u >= 0: the lower end of u*p uses u.lo if p.lo >= 0 else u.hi; the upper end likewise
    double ul = (p.lo >= 0.0) ? u.lo : u.hi;
    double uh = (p.hi >= 0.0) ? u.hi : u.lo;
    return {__fma_rd(ul, p.lo, clo), __fma_ru(uh, p.hi, chi)};
}

// Enclosures of sin x and cos x for x in [x.lo, x.hi], 0 <= x.lo <= x.hi <= pi/4 + 2^-60.
MB_DEV void iv_sincos(const Ival &x, Ival &s, Ival &c) {
    const Ival u{__dmul_rd(x.lo, x.lo), __dmul_ru(x.hi, x.hi)};
    Ival p{CERT_S_LO[8], CERT_S_HI[8]};
#pragma unroll
    for (int k = 7; k >= 0; --k) p = horner_step(u, p, CERT_S_LO[k], CERT_S_HI[k]);
    // sin x / x >= 0.9 > 0 on this range
    s = {__dmul_rd(x.lo, p.lo), __dmul_ru(x.hi, p.hi)};
    double xp = x.hi;                              // x^19 rounded up
#pragma unroll
    for (int k = 0; k < 9; ++k) xp = __dmul_ru(xp, u.hi);
    const double rs = __dmul_ru(xp, CERT_REM_S);
    s.lo = __dsub_rd(s.lo, rs);
    s.hi = __dadd_ru(s.hi, rs);
    Ival q{CERT_C_LO[9], CERT_C_HI[9]};
#pragma unroll
    for (int k = 8; k >= 0; --k) q = horner_step(u, q, CERT_C_LO[k], CERT_C_HI[k]);
    double up = u.hi;                              // x^20 rounded up
#pragma unroll
    for (int k = 0; k < 9; ++k) up = __dmul_ru(up, u.hi);
    const double rc = __dmul_ru(up, CERT_REM_C);
    c = {__dsub_rd(q.lo, rc), __dadd_ru(q.hi, rc)};
}

MB_DEV Ival iv_neg(const Ival &a) { return {-a.hi, -a.lo}; }

// point * interval
MB_DEV Ival iv_scale(double a, const Ival &b) {
    return a >= 0.0 ? Ival{__dmul_rd(a, b.lo), __dmul_ru(a, b.hi)} : Ival{__dmul_rd(a, b.hi), __dmul_ru(a, b.lo)};
}

// non-negative interval w times interval a
MB_DEV Ival iv_wmul(const Ival &w, const Ival &a) {
    double lo = a.lo >= 0.0 ? __dmul_rd(w.lo, a.lo) : __dmul_rd(w.hi, a.lo);
    double hi = a.hi >= 0.0 ? __dmul_ru(w.hi, a.hi) : __dmul_ru(w.lo, a.hi);
    return {lo, hi};
}

// Enclosure of exp(-y) for y in [ylo, yhi], 0 <= ylo <= yhi.
MB_DEV Ival iv_exp_neg(double ylo, double yhi) {
    const double e_small = exp(-yhi), e_big = exp(-ylo);
    const double tiny = 4.0 * 4.9406564584124654e-324;     // absolute slack in the subnormal range
    double lo = __dmul_rd(e_small, 1.0 - 4.440892098500626e-16);
    double hi = __dmul_ru(e_big, 1.0 + 4.440892098500626e-16);
    if (e_small < 2.2250738585072014e-308) lo = fmax(0.0, __dsub_rd(lo, tiny));
    if (e_big < 2.2250738585072014e-308) hi = __dadd_ru(hi, tiny);
    return {lo, hi};
}

struct CertTerm {
    Ival t;         // 2 w Re(c e^{i theta})
    double abs_hi;  // 2 w |c| rounded up
    Ival dd, dk;    // -2 w gamma Im(c e^{i theta}) and -2 w gamma^2 Re(c e^{i theta}) (GRAD only)
};

// -2 x for an interval x (exact)
MB_DEV Ival iv_m2(const Ival &x) { return {-2.0 * x.hi, -2.0 * x.lo}; }

// Term j; k lies in [k_lo, k_hi]; term_rad (nullable) is the per-term radius at index jr.  With
// GRAD the term's derivatives in v (= delta) and k are enclosed too:
//   d/dv 2 w Re(c e^{i gamma v}) = -2 w gamma Im(c e^{i gamma v}) = -2 w gamma (Re c sin + Im c cos),
//   d/dk 2 w Re(c e^{i gamma v}) = -2 w gamma^2 Re(c e^{i gamma v}),
// from the same sine/cosine and weight intervals and gamma in [gamma_lo, gamma_hi]; a radius rho
// of c e^{i gamma v} (|c| gamma_hi v_rad + term_rad) widens them by 2 w_hi gamma_hi rho and
// 2 w_hi gamma_hi^2 rho (each derivative in v brings one more factor gamma).
template <bool GRAD>
MB_DEV CertTerm cert_term(const TabView &tv, int64_t j, uint64_t vi, uint64_t vf, double k_lo, double k_hi,
                          double v_rad, const double *term_rad, int64_t jr) {
    uint64_t hi, lo;
    phase128_exact((uint32_t)vf, (uint32_t)(vf >> 32), (uint32_t)vi, (uint32_t)(vi >> 32), tv.g0[j], tv.g1[j],
                   tv.g2[j], tv.g3[j], tv.g4[j], hi, lo);
    const int q = (int)(hi >> 62);
    const uint64_t m = hi & ((1ull << 62) - 1);
    const double two_m62 = 2.168404344971009e-19;
    Ival r{__ull2double_rd(m) * two_m62, __ull2double_ru(m + 1) * two_m62};
    bool swap = false;
    if (r.lo >= 0.5) {
        r = {__dsub_rd(1.0, r.hi), __dsub_ru(1.0, r.lo)};
        swap = true;
    }
    const Ival x{__dmul_rd(CERT_PIO2_LO, r.lo), __dmul_ru(CERT_PIO2_HI, r.hi)};
    Ival s, c;
    iv_sincos(x, s, c);
    if (swap) {
        Ival t = s;
        s = c;
        c = t;
    }
    // rotate by q quarter turns: q=0 (s,c) 1 (c,-s) 2 (-s,-c) 3 (-c,s)
    Ival S, Cc;
    switch (q) {
        case 0: S = s; Cc = c; break;
        case 1: S = c; Cc = iv_neg(s); break;
        case 2: S = iv_neg(s); Cc = iv_neg(c); break;
        default: S = iv_neg(c); Cc = s; break;
    }
    const double cr = tv.cre[j], ci = tv.cim[j];
    const Ival a1 = iv_scale(cr, Cc), a2 = iv_scale(ci, S);
    const Ival A{__dsub_rd(a1.lo, a2.hi), __dsub_ru(a1.hi, a2.lo)};
    const double g = tv.gamma[j];
    const double glo = __dmul_rd(g, 1.0 - 8.881784197001252e-16), ghi = __dmul_ru(g, 1.0 + 8.881784197001252e-16);
    const double ylo = __dmul_rd(__dmul_rd(k_lo, glo), glo), yhi = __dmul_ru(__dmul_ru(k_hi, ghi), ghi);
    const Ival w = iv_exp_neg(ylo, yhi);
    Ival t = iv_wmul(w, A);
    t.lo *= 2.0;
    t.hi *= 2.0;
    const double cabs = __dsqrt_ru(__fma_ru(cr, cr, __dmul_ru(ci, ci)));
    double rad = 0.0;
    if (v_rad > 0.0) rad = __dmul_ru(__dmul_ru(cabs, ghi), v_rad);
    if (term_rad) rad = __dadd_ru(rad, term_rad[jr]);
    double wr = 0.0;
    if (rad > 0.0) {
        wr = __dmul_ru(2.0 * w.hi, rad);
        t.lo = __dsub_rd(t.lo, wr);
        t.hi = __dadd_ru(t.hi, wr);
    }
    CertTerm out{t, __dmul_ru(2.0 * w.hi, cabs), {0.0, 0.0}, {0.0, 0.0}};
    if constexpr (GRAD) {
        const Ival b1 = iv_scale(cr, S), b2 = iv_scale(ci, Cc);
        const Ival B{__dadd_rd(b1.lo, b2.lo), __dadd_ru(b1.hi, b2.hi)};     // Im(c e^{i theta})
        const Ival wg{__dmul_rd(w.lo, glo), __dmul_ru(w.hi, ghi)};          // w gamma >= 0
        const Ival wg2{__dmul_rd(wg.lo, glo), __dmul_ru(wg.hi, ghi)};      // w gamma^2 >= 0
        out.dd = iv_m2(iv_wmul(wg, B));
        out.dk = iv_m2(iv_wmul(wg2, A));
        if (wr > 0.0) {
            const double r1 = __dmul_ru(wr, ghi), r2 = __dmul_ru(r1, ghi);
            out.dd = {__dsub_rd(out.dd.lo, r1), __dadd_ru(out.dd.hi, r1)};
            out.dk = {__dsub_rd(out.dk.lo, r2), __dadd_ru(out.dk.hi, r2)};
        }
    }
    return out;
}

constexpr int CERT_THREADS = 256;

// Number of sums per (block, candidate): lo/hi of K2 and abs_hi, plus lo/hi of both derivatives.
template <bool GRAD>
__host__ __device__ constexpr int cert_sums() { return GRAD ? 7 : 3; }

// grid (zero blocks, candidates); partial[(blockIdx.x * P + p) * NS + s] with s = K2 lo, K2 hi,
// abs_hi[, dd lo, dd hi, dk lo, dk hi]: lower ends summed with __dadd_rd, upper ends with __dadd_ru.
template <bool GRAD>
__global__ void __launch_bounds__(CERT_THREADS)
k2_certified_kernel(TabView tv, const uint64_t *vi, const uint64_t *vf, const double *v_rad, int64_t P, int64_t j0,
                    int64_t j1, double k_lo, double k_hi, const double *term_rad, double *partial) {
    constexpr int NS = cert_sums<GRAD>();
    const int64_t p = blockIdx.y;
    const uint64_t a = vi[p], b = vf[p];
    const double vr = v_rad ? v_rad[p] : 0.0;
    double acc[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) acc[q] = 0.0;
    for (int64_t jr = (int64_t)blockIdx.x * CERT_THREADS + threadIdx.x; j0 + jr < j1; jr += (int64_t)gridDim.x * CERT_THREADS) {
        CertTerm ct = cert_term<GRAD>(tv, j0 + jr, a, b, k_lo, k_hi, vr, term_rad, jr);
        acc[0] = __dadd_rd(acc[0], ct.t.lo);
        acc[1] = __dadd_ru(acc[1], ct.t.hi);
        acc[2] = __dadd_ru(acc[2], ct.abs_hi);
        if constexpr (GRAD) {
            acc[3] = __dadd_rd(acc[3], ct.dd.lo);
            acc[4] = __dadd_ru(acc[4], ct.dd.hi);
            acc[5] = __dadd_rd(acc[5], ct.dk.lo);
            acc[6] = __dadd_ru(acc[6], ct.dk.hi);
        }
    }
    // lower ends (even indices except abs_hi at 2) round down, the others up
    auto up = [](int q) { return q == 1 || q == 2 || q == 4 || q == 6; };
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            const double x = __shfl_xor_sync(0xffffffffu, acc[q], o);
            acc[q] = up(q) ? __dadd_ru(acc[q], x) : __dadd_rd(acc[q], x);
        }
    }
    __shared__ double red[CERT_THREADS / 32][NS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NS; ++q) red[warp][q] = acc[q];
    __syncthreads();
    if (threadIdx.x == 0) {
        double *o = partial + ((int64_t)blockIdx.x * P + p) * NS;
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            double v = 0.0;
            for (int w = 0; w < CERT_THREADS / 32; ++w) v = up(q) ? __dadd_ru(v, red[w][q]) : __dadd_rd(v, red[w][q]);
            o[q] = v;
        }
    }
}

// out[s * P + p] for the NS sums of candidate p (the same order as the partials).
template <bool GRAD>
__global__ void certified_reduce_kernel(const double *partial, int64_t P, int nblk, double *out) {
    constexpr int NS = cert_sums<GRAD>();
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
#pragma unroll
    for (int q = 0; q < NS; ++q) {
        const bool up = q == 1 || q == 2 || q == 4 || q == 6;
        double v = 0.0;
        for (int b = 0; b < nblk; ++b) {
            const double x = partial[((int64_t)b * P + p) * NS + q];
            v = up ? __dadd_ru(v, x) : __dadd_rd(v, x);
        }
        out[q * P + p] = v;
    }
}

// out (device, NS x P): rows K2 lo, K2 hi, abs_hi [, dd lo, dd hi, dk lo, dk hi].
int launch_certified(Table &t, const uint64_t *d_vi, const uint64_t *d_vf, const double *d_vrad, int64_t P,
                     int64_t j0, int64_t j1, double k_lo, double k_hi, const double *d_term_rad, bool grad,
                     double *d_out, cudaStream_t s) {
    if (P == 0) return MB_OK;
    const int64_t n_use = std::max<int64_t>(0, j1 - j0);
    int sms = 148;
    MB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, t.device));
    int64_t want = std::max<int64_t>(1, ((int64_t)sms * 8 + P - 1) / P);
    int64_t nblk = std::max<int64_t>(1, std::min(want, (n_use + CERT_THREADS - 1) / CERT_THREADS));
    MB_CHECK_ARG(P <= 65535, "certified: P=%lld exceeds 65535 candidates per call", (long long)P);
    const int ns = grad ? cert_sums<true>() : cert_sums<false>();
    MB_TRY(t.work.ensure((size_t)nblk * P * ns * sizeof(double)));
    double *partial = (double *)t.work.p;
    dim3 grid((unsigned)nblk, (unsigned)P);
    const unsigned rgrid = (unsigned)((P + 255) / 256);
    if (grad) {
        k2_certified_kernel<true><<<grid, CERT_THREADS, 0, s>>>(view(t), d_vi, d_vf, d_vrad, P, j0, j1, k_lo, k_hi,
                                                                d_term_rad, partial);
        MB_CUDA(cudaGetLastError());
        certified_reduce_kernel<true><<<rgrid, 256, 0, s>>>(partial, P, (int)nblk, d_out);
    } else {
        k2_certified_kernel<false><<<grid, CERT_THREADS, 0, s>>>(view(t), d_vi, d_vf, d_vrad, P, j0, j1, k_lo, k_hi,
                                                                 d_term_rad, partial);
        MB_CUDA(cudaGetLastError());
        certified_reduce_kernel<false><<<rgrid, 256, 0, s>>>(partial, P, (int)nblk, d_out);
    }
    MB_CUDA(cudaGetLastError());
    return MB_OK;
}

}  // namespace mb

using namespace mb;

namespace {

// The shared body of the certified entry points: checks, staging, launch, copy-out of
// out_rows[r] (host, P each) from the NS device rows (null entries are skipped).
int certified_call(const char *who, mb_table *h, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                   const double *v_rad, double k_lo, double k_hi, int64_t j0, int64_t j1, const double *term_rad,
                   bool grad, double *const *out_rows) {
    MB_CHECK_ARG(h && v_int && v_frac, "%s: null argument", who);
    MB_CHECK_ARG(P >= 0 && P <= 65535, "%s: P=%lld out of range (0..65535)", who, (long long)P);
    MB_CHECK_ARG(std::isfinite(k_lo) && std::isfinite(k_hi) && 0.0 <= k_lo && k_lo <= k_hi,
                 "%s: k interval [%g, %g]", who, k_lo, k_hi);
    if (P == 0) return MB_OK;
    Table &t = table_of(h);
    MB_CHECK_ARG(0 <= j0 && j0 <= j1 && j1 <= t.n, "%s: zero range [%lld, %lld) of %lld", who, (long long)j0,
                 (long long)j1, (long long)t.n);
    const int64_t n_use = j1 - j0;
    if (v_rad)
        for (int64_t p = 0; p < P; ++p)
            MB_CHECK_ARG(std::isfinite(v_rad[p]) && v_rad[p] >= 0.0, "%s: v_rad[%lld]", who, (long long)p);
    if (term_rad)
        for (int64_t j = 0; j < n_use; ++j)
            MB_CHECK_ARG(std::isfinite(term_rad[j]) && term_rad[j] >= 0.0, "%s: term_rad[%lld]", who, (long long)j);
    MB_TRY(device_guard(t.device));
    const int ns = grad ? cert_sums<true>() : cert_sums<false>();
    const size_t cb = (size_t)P * 8, rb = term_rad ? (size_t)n_use * 8 : 0;
    MB_TRY(t.io.ensure((3 + ns) * cb + rb + 256));
    char *base = (char *)t.io.p;
    uint64_t *d_vi = (uint64_t *)base, *d_vf = (uint64_t *)(base + cb);
    double *d_vrad = (double *)(base + 2 * cb), *d_out = (double *)(base + 3 * cb);
    double *d_rad = term_rad ? (double *)(base + (3 + ns) * cb) : nullptr;
    MB_CUDA(cudaMemcpyAsync(d_vi, v_int, cb, cudaMemcpyHostToDevice, t.stream));
    MB_CUDA(cudaMemcpyAsync(d_vf, v_frac, cb, cudaMemcpyHostToDevice, t.stream));
    if (v_rad) MB_CUDA(cudaMemcpyAsync(d_vrad, v_rad, cb, cudaMemcpyHostToDevice, t.stream));
    if (term_rad && rb) MB_CUDA(cudaMemcpyAsync(d_rad, term_rad, rb, cudaMemcpyHostToDevice, t.stream));
    MB_TRY(launch_certified(t, d_vi, d_vf, v_rad ? d_vrad : nullptr, P, j0, j1, k_lo, k_hi, d_rad, grad, d_out,
                            t.stream));
    for (int r = 0; r < ns; ++r)
        if (out_rows[r]) MB_CUDA(cudaMemcpyAsync(out_rows[r], d_out + r * P, cb, cudaMemcpyDeviceToHost, t.stream));
    MB_CUDA(cudaStreamSynchronize(t.stream));
    return MB_OK;
}

}  // namespace

extern "C" int mb_k2_certified_range(mb_table *h, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                                     const double *v_rad, double k_lo, double k_hi, int64_t j0, int64_t j1,
                                     const double *term_rad, double *out_lo, double *out_hi, double *out_abs_hi) {
    MB_CHECK_ARG(out_lo && out_hi, "mb_k2_certified_range: null argument");
    double *rows[3] = {out_lo, out_hi, out_abs_hi};
    return certified_call("mb_k2_certified_range", h, P, v_int, v_frac, v_rad, k_lo, k_hi, j0, j1, term_rad, false,
                          rows);
}

extern "C" int mb_k2_certified_grad_range(mb_table *h, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                                          const double *v_rad, double k_lo, double k_hi, int64_t j0, int64_t j1,
                                          const double *term_rad, double *out_lo, double *out_hi) {
    MB_CHECK_ARG(out_lo && out_hi, "mb_k2_certified_grad_range: null argument");
    double *rows[7] = {out_lo, out_hi, nullptr, out_lo + P, out_hi + P, out_lo + 2 * P, out_hi + 2 * P};
    return certified_call("mb_k2_certified_grad_range", h, P, v_int, v_frac, v_rad, k_lo, k_hi, j0, j1, term_rad,
                          true, rows);
}

extern "C" int mb_k2_certified(mb_table *h, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                               const double *v_rad, double k, double T, const double *term_rad,
                               double *out_lo, double *out_hi, double *out_abs_hi) {
    MB_CHECK_ARG(h, "mb_k2_certified: null table");
    MB_CHECK_ARG(std::isfinite(k) && k >= 0.0, "mb_k2_certified: k=%g", k);
    MB_CHECK_ARG(!std::isnan(T), "mb_k2_certified: T is NaN");
    return mb_k2_certified_range(h, P, v_int, v_frac, v_rad, k, k, 0, table_of(h).count_below(T), term_rad, out_lo,
                                 out_hi, out_abs_hi);
}
