// Per-peak polish of  h(ddy) = sum_j w_j (A_j cos(gamma_j ddy) - B_j sin(gamma_j ddy)),
// one thread-block cluster of POLISH_CLUSTER CTAs per peak: each CTA sums a stride of the zeros,
// and the sequential steps of the reference loops become cluster-wide reductions through
// distributed shared memory (every CTA adds the CTA totals in rank order, so all CTAs hold the
// same bits and take the same branches).  A handful of peaks thus spreads over 8x as many SMs.
//
// (A_j, B_j) = 2 c_j e^{i gamma_j y} of a peak come from a source:
//   ABMatrix  rows of caller matrices (the reference's A/B contract, search/path1_eval_fast.cpp:15-53,
//             search/path1_kernel_opt.py:71-91), row-major with row stride ld;
//   ABExact   computed on the fly from the exact 128-bit phase of the peak's v (+ delta), so no
//             P x N matrix is written or read.
#pragma once
#include <cooperative_groups.h>

#include "k2_common.cuh"
#include "k2_internal.h"

namespace mb {

constexpr int POLISH_THREADS = 256;
constexpr int POLISH_CLUSTER = 8;     // CTAs per peak (portable cluster size)
constexpr int64_t POLISH_STRIDE = (int64_t)POLISH_CLUSTER * POLISH_THREADS;

// Sum over the CTA; every thread gets the result.  Warp partials are added in warp order, so the
// result does not depend on scheduling.
__device__ __forceinline__ double block_sum(double x, double *red) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = x;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < POLISH_THREADS / 32; ++w) s += red[w];
    return s;
}

// The calling thread's place in its peak's cluster and the cluster-wide sum.
struct Team {
    int64_t first;         // rank * POLISH_THREADS + threadIdx.x: first zero of this thread
    double *red;           // CTA scratch of block_sum
    double *slot;          // this CTA's two exchange slots (double-buffered)
    int parity;
    double *redv = nullptr;    // sumv scratch: [POLISH_THREADS / 32][N]
    double *slotv = nullptr;   // sumv exchange slots: [2][N], double-buffered by vparity
    int vparity = 0;

    // Cluster-wide sums of N values with one block reduction and one cluster barrier; each value
    // is added in exactly the order of sum() (warp shuffle tree, warps in order, ranks in order),
    // so the results are the bits of N separate sum() calls.
    template <int N>
    __device__ void sumv(double (&x)[N]) {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
        for (int i = 0; i < N; ++i)
            for (int o = 16; o > 0; o >>= 1) x[i] += __shfl_xor_sync(0xffffffffu, x[i], o);
        __syncthreads();
        if (lane == 0)
#pragma unroll
            for (int i = 0; i < N; ++i) redv[warp * N + i] = x[i];
        __syncthreads();
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double t = 0.0;
#pragma unroll
            for (int w = 0; w < POLISH_THREADS / 32; ++w) t += redv[w * N + i];
            x[i] = t;
        }
        namespace cg = cooperative_groups;
        cg::cluster_group cl = cg::this_cluster();
        if (threadIdx.x == 0)
#pragma unroll
            for (int i = 0; i < N; ++i) slotv[vparity * N + i] = x[i];
        cl.sync();
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double t = 0.0;
#pragma unroll
            for (int r = 0; r < POLISH_CLUSTER; ++r) t += *cl.map_shared_rank(&slotv[vparity * N + i], r);
            x[i] = t;
        }
        vparity ^= 1;
    }

    // Sum of x over all threads of the cluster; every thread of every CTA gets the same value.
    // One cluster barrier per call: a CTA rewrites a slot only after the barrier of the next
    // call, which every peer reaches after reading it.
    __device__ double sum(double x) {
        const double s = block_sum(x, red);
        namespace cg = cooperative_groups;
        cg::cluster_group cl = cg::this_cluster();
        if (threadIdx.x == 0) slot[parity] = s;
        cl.sync();
        double t = 0.0;
#pragma unroll
        for (int r = 0; r < POLISH_CLUSTER; ++r) t += *cl.map_shared_rank(&slot[parity], r);
        parity ^= 1;
        return t;
    }
};

struct ABMatrix {
    // zeros per iteration of the polish loops: the passes over a matrix are bound by global-load
    // latency, so each iteration issues the loads of ZPI zeros before computing any of them
    // (2: -20 % time at 64 registers; 3 spills, 4 takes 76 registers and is slower)
    static constexpr int ZPI = 2;
    const double *A, *B;
    int64_t ld;
    struct Peak {
        const double *a, *b;
    };
    MB_DEV Peak peak(int64_t p) const { return Peak{A + p * ld, B + p * ld}; }
    MB_DEV void at(const Peak &pk, int64_t j, double &a, double &b) const {
        a = pk.a[j];
        b = pk.b[j];
    }
};

MB_DEV void two_sum(double a, double b, double &s, double &e) {
    s = a + b;
    double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

// Exact-phase (A_j, B_j) of y = v + delta:
//   turns = frac(v G_j) [exact, 128 bits] + frac(delta G_j) [delta g_int exact by two-product,
//   delta frac(G_j) rounded once], summed in double-double and reduced to [-1/2, 1/2];
//   sin/cos(2 pi turns) = sincospi of the leading part, corrected to first order by the trailing
//   part.  The angle error is below 2pi (|delta| 2^-52 + 2^-100) rad, so A and B carry the FP64
//   rounding of sincospi and of 2 (c_re cos - c_im sin) only.  Requires |delta| <= 2^16.
struct ABExact {
    static constexpr int ZPI = 1;   // compute bound: one zero per iteration (more would spill)
    TabView t;
    const uint64_t *vi, *vf;
    const double *delta;   // may be null
    struct Peak {
        uint32_t v0, v1, v2, v3;
        double d;
    };
    MB_DEV Peak peak(int64_t p) const {
        Peak k;
        const uint64_t a = vi[p], b = vf[p];
        k.v0 = (uint32_t)b;
        k.v1 = (uint32_t)(b >> 32);
        k.v2 = (uint32_t)a;
        k.v3 = (uint32_t)(a >> 32);
        k.d = delta ? delta[p] : 0.0;
        return k;
    }
    MB_DEV void at(const Peak &pk, int64_t j, double &A, double &B) const {
        const uint32_t g0 = t.g0[j], g1 = t.g1[j], g2 = t.g2[j], g3 = t.g3[j], g4 = t.g4[j];
        uint64_t hi, lo;
        phase128_exact(pk.v0, pk.v1, pk.v2, pk.v3, g0, g1, g2, g3, g4, hi, lo);
        // frac(v G) as signed turns: hi = [s32 | u32] exactly, lo below 2^-64
        const double a = s32_to_f64((int32_t)(uint32_t)(hi >> 32)) * 0x1p-32;
        const double b = u32_to_f64((uint32_t)hi) * 0x1p-64;
        const double c = (double)lo * 0x1p-128;
        double s, e;
        two_sum(a, b, s, e);
        e += c;
        if (pk.d != 0.0) {
            const double gi = u32_to_f64(g4);
            double p = pk.d * gi;
            const double pe = fma(pk.d, gi, -p);                   // exact product remainder
            p -= rint(p);                                           // exact for |p| < 2^52
            const double f = fma(u32_to_f64(g3), 0x1p-32, fma(u32_to_f64(g2), 0x1p-64, u32_to_f64(g1) * 0x1p-96));
            double e2, e3;
            two_sum(s, p, s, e2);
            two_sum(s, pk.d * f, s, e3);
            e += e2 + e3 + pe;
        }
        s -= rint(s);                                               // exact; |s| <= 1/2
        double sn, cs;
        sincospi(2.0 * s, &sn, &cs);
        const double eps = 6.283185307179586 * e;
        const double sn2 = fma(eps, cs, sn);
        const double cs2 = fma(-eps, sn, cs);
        const double cr = t.cre[j], ci = t.cim[j];
        A = 2.0 * fma(cr, cs2, -ci * sn2);
        B = 2.0 * fma(cr, sn2, ci * cs2);
    }
};

// h at ddy (all threads get it).
template <class Src>
__device__ double polish_h(const Src &src, const typename Src::Peak &pk, int64_t n, const double *gamma,
                           const double *w, double ddy, Team &tm) {
    constexpr int Z = Src::ZPI;
    double h = 0.0;
    for (int64_t i = tm.first; i < n; i += Z * POLISH_STRIDE) {
        double a[Z], b[Z], g[Z], wv[Z];
#pragma unroll
        for (int z = 0; z < Z; ++z) {
            const int64_t iz = i + z * POLISH_STRIDE;
            a[z] = b[z] = g[z] = wv[z] = 0.0;
            if (z == 0 || iz < n) {
                src.at(pk, iz, a[z], b[z]);
                g[z] = gamma[iz];
                wv[z] = w[iz];
            }
        }
        // the terms in zero order, as with one zero per iteration
#pragma unroll
        for (int z = 0; z < Z; ++z) {
            if (z > 0 && i + z * POLISH_STRIDE >= n) break;
            double sn, cs;
            sincos(g[z] * ddy, &sn, &cs);
            h += wv[z] * (a[z] * cs - b[z] * sn);
        }
    }
    return tm.sum(h);
}

// Newton on h'(ddy) = 0 from ddy: at most `iters` steps, each clamped to +-clamp; stops after a
// step below step_tol or when |h''| <= 1e-12 (search/path1_eval_fast.cpp:103-129,
// search/path1_kernel_opt.py:125-138 and :197-212 differ only in these three constants).
template <class Src>
__device__ double polish_newton(const Src &src, const typename Src::Peak &pk, int64_t n, const double *gamma,
                                const double *w, double ddy, int iters, double clamp, double step_tol,
                                Team &tm) {
    for (int it = 0; it < iters; ++it) {
        constexpr int Z = Src::ZPI;
        double fp = 0.0, fpp = 0.0;
        for (int64_t i = tm.first; i < n; i += Z * POLISH_STRIDE) {
            double a[Z], b[Z], g[Z], wv[Z];
#pragma unroll
            for (int z = 0; z < Z; ++z) {
                const int64_t iz = i + z * POLISH_STRIDE;
                a[z] = b[z] = g[z] = wv[z] = 0.0;
                if (z == 0 || iz < n) {
                    src.at(pk, iz, a[z], b[z]);
                    g[z] = gamma[iz];
                    wv[z] = w[iz];
                }
            }
#pragma unroll
            for (int z = 0; z < Z; ++z) {
                if (z > 0 && i + z * POLISH_STRIDE >= n) break;
                double sn, cs;
                sincos(g[z] * ddy, &sn, &cs);
                const double val = a[z] * cs - b[z] * sn;
                const double dval = g[z] * (-a[z] * sn - b[z] * cs);
                fp += wv[z] * dval;
                fpp += wv[z] * (-(g[z] * g[z]) * val);
            }
        }
        fp = tm.sum(fp);
        fpp = tm.sum(fpp);
        if (!(fabs(fpp) > 1e-12)) break;
        double step = fp / fpp;
        step = fmin(fmax(step, -clamp), clamp);
        ddy -= step;
        if (fabs(step) < step_tol) break;
    }
    return ddy;
}

// Polish modes (the three reference loops).
enum PolishMode : int {
    // search/path1_eval_fast.cpp:76-141: grid m = -steps..steps, ddy = (hw m)/steps, over the first
    // min(n, 4096) zeros, best starts at |h0| (strict >); Newton from the best point (6 steps,
    // clamp 1e-4, stop below 1e-13); keep h0 if |h0| > |h_final|.
    POLISH_EVAL_FAST = 0,
    // search/path1_kernel_opt.py:94-147: grid ddys[m] (caller array, numpy linspace) over all n
    // zeros, first argmax of |h|; Newton (8 steps, clamp 2e-5, stop below 1e-14) from 0 and from
    // the grid's best; keep a start's h only if |h| > |best so far| (best starts at h0, ddy 0).
    POLISH_SINGLE = 1,
    // search/path1_kernel_opt.py:193-219: Newton (4 steps, clamp 1e-5, stop below 1e-13) from
    // ddy_pol[p]; keep (h, ddy) if |h| > |h_unpol[p]|, else (h_unpol[p], 0).
    POLISH_TOPK = 2,
};

struct PolishArgs {
    int64_t n;                    // zeros summed
    const double *gamma, *w;
    const double *grid;           // POLISH_SINGLE: ddy values; else null
    int n_grid;                   // POLISH_SINGLE: grid size; POLISH_EVAL_FAST: grid_steps
    double half;                  // POLISH_EVAL_FAST: grid half width
    const int *sel;               // POLISH_TOPK: peak index of each CTA; else null (CTA = peak)
    double *h_unpol, *h_pol, *ddy_pol;
};

// Grid: POLISH_CLUSTER CTAs per peak (cluster c serves peak sel[c], or c).  Rank 0 writes the
// results; every CTA waits at a last cluster barrier so none exits while a peer may still read
// its exchange slots.
template <class Src, int MODE>
__global__ void __cluster_dims__(POLISH_CLUSTER, 1, 1) __launch_bounds__(POLISH_THREADS)
    peak_polish_kernel(Src src, PolishArgs a) {
    __shared__ double red[POLISH_THREADS / 32];
    __shared__ double slot[2];
    namespace cg = cooperative_groups;
    const int rank = (int)cg::this_cluster().block_rank();
    const int64_t cid = blockIdx.x / POLISH_CLUSTER;
    Team tm{(int64_t)rank * POLISH_THREADS + threadIdx.x, red, slot, 0};
    const bool writer = rank == 0 && threadIdx.x == 0;
    const int64_t p = a.sel ? a.sel[cid] : cid;
    const typename Src::Peak pk = src.peak(p);
    const int64_t n = a.n;
    if (MODE == POLISH_TOPK) {
        const double hu = a.h_unpol[p];
        const double ddy = polish_newton(src, pk, n, a.gamma, a.w, a.ddy_pol[p], 4, 1e-5, 1e-13, tm);
        const double h = polish_h(src, pk, n, a.gamma, a.w, ddy, tm);
        if (writer) {
            const bool better = fabs(h) > fabs(hu);
            a.h_pol[p] = better ? h : hu;
            a.ddy_pol[p] = better ? ddy : 0.0;
        }
    } else {
        constexpr int Z = Src::ZPI;
        double s = 0.0;
        for (int64_t i = tm.first; i < n; i += Z * POLISH_STRIDE) {
            double x[Z], wv[Z];
#pragma unroll
            for (int z = 0; z < Z; ++z) {
                const int64_t iz = i + z * POLISH_STRIDE;
                x[z] = wv[z] = 0.0;
                if (z == 0 || iz < n) {
                    double y;
                    src.at(pk, iz, x[z], y);
                    wv[z] = a.w[iz];
                }
            }
#pragma unroll
            for (int z = 0; z < Z; ++z)
                if (z == 0 || i + z * POLISH_STRIDE < n) s += wv[z] * x[z];
        }
        const double h0 = tm.sum(s);
        if (MODE == POLISH_EVAL_FAST) {
            const int steps = a.n_grid;
            const int64_t k_scan = n < 4096 ? n : 4096;
            double best_ddy = 0.0, best_abs = fabs(h0);
            for (int m = -steps; m <= steps && steps > 0; ++m) {
                const double ddy = (a.half * m) / steps;
                const double hs = fabs(polish_h(src, pk, k_scan, a.gamma, a.w, ddy, tm));
                if (hs > best_abs) {
                    best_abs = hs;
                    best_ddy = ddy;
                }
            }
            const double ddy = polish_newton(src, pk, n, a.gamma, a.w, best_ddy, 6, 1e-4, 1e-13, tm);
            const double hf = polish_h(src, pk, n, a.gamma, a.w, ddy, tm);
            if (writer) {
                a.h_unpol[p] = h0;
                const bool keep0 = fabs(h0) > fabs(hf);
                a.h_pol[p] = keep0 ? h0 : hf;
                a.ddy_pol[p] = keep0 ? 0.0 : ddy;
            }
        } else {  // POLISH_SINGLE
            double best_h = h0, best_ddy = 0.0;
            int n_starts = 1;
            double grid_best = 0.0;
            if (a.n_grid > 0) {
                double top = -1.0;
                for (int m = 0; m < a.n_grid; ++m) {
                    const double hs = fabs(polish_h(src, pk, n, a.gamma, a.w, a.grid[m], tm));
                    if (hs > top) {
                        top = hs;
                        grid_best = a.grid[m];
                    }
                }
                n_starts = 2;
            }
            for (int st = 0; st < n_starts; ++st) {
                const double ddy =
                    polish_newton(src, pk, n, a.gamma, a.w, st == 0 ? 0.0 : grid_best, 8, 2e-5, 1e-14, tm);
                const double h = polish_h(src, pk, n, a.gamma, a.w, ddy, tm);
                if (fabs(h) > fabs(best_h)) {
                    best_h = h;
                    best_ddy = ddy;
                }
            }
            if (writer) {
                a.h_unpol[p] = h0;
                a.h_pol[p] = best_h;
                a.ddy_pol[p] = best_ddy;
            }
        }
    }
    cg::this_cluster().sync();
}

// Degree-16 Taylor moments of h around ddy = 0 and their grid maximum
// (search/path1_kernel_opt.py:150-191): u = gamma 1e-4, z = ddy 1e4,
//   C_m = sum_j w_j A_j u_j^{2m} (-1)^m/(2m)!      m = 0..8
//   S_m = sum_j w_j B_j u_j^{2m+1} (-1)^m/(2m+1)!  m = 0..7
//   h(z) = sum_m C_m z^{2m} - sum_m S_m z^{2m+1};   h_unpol = C_0; h_pol, ddy_pol = the first
//   grid point of largest |h(z)|.  The moments are accumulated per thread and reduced over the
//   CTA (the reference's two GEMMs, here one pass over the peak's terms).
struct MomentArgs {
    int64_t n;
    const double *gamma, *w;
    const double *grid;
    int n_grid;
    double *h_unpol, *h_pol, *ddy_pol;
};

template <class Src>
__global__ void __cluster_dims__(POLISH_CLUSTER, 1, 1) __launch_bounds__(POLISH_THREADS)
    taylor_moments_kernel(Src src, MomentArgs a) {
    __shared__ double red[POLISH_THREADS / 32];
    __shared__ double slot[2];
    __shared__ double mom[17];
    __shared__ double best_v[POLISH_THREADS], best_h[POLISH_THREADS];
    __shared__ int best_i[POLISH_THREADS];
    __shared__ double redv[(POLISH_THREADS / 32) * 17], slotv[2 * 17];
    namespace cg = cooperative_groups;
    const int rank = (int)cg::this_cluster().block_rank();
    Team tm{(int64_t)rank * POLISH_THREADS + threadIdx.x, red, slot, 0, redv, slotv, 0};
    const int64_t p = blockIdx.x / POLISH_CLUSTER;
    const typename Src::Peak pk = src.peak(p);
    // (-1)^m/(2m)! and (-1)^m/(2m+1)!
    constexpr double CC[9] = {1.0, -1.0 / 2, 1.0 / 24, -1.0 / 720, 1.0 / 40320, -1.0 / 3628800,
                              1.0 / 479001600, -1.0 / 87178291200.0, 1.0 / 20922789888000.0};
    constexpr double CS[8] = {1.0, -1.0 / 6, 1.0 / 120, -1.0 / 5040, 1.0 / 362880, -1.0 / 39916800,
                              1.0 / 6227020800.0, -1.0 / 1307674368000.0};
    double c[9], s[8];
#pragma unroll
    for (int m = 0; m < 9; ++m) c[m] = 0.0;
#pragma unroll
    for (int m = 0; m < 8; ++m) s[m] = 0.0;
    for (int64_t i = tm.first; i < a.n; i += POLISH_STRIDE) {
        double x, y;
        src.at(pk, i, x, y);
        const double u = a.gamma[i] * 1.0e-4, u2 = u * u;
        const double wa = a.w[i] * x, wb = a.w[i] * y * u;
        double pw = 1.0;
#pragma unroll
        for (int m = 0; m < 9; ++m) {
            c[m] = fma(wa * pw, CC[m], c[m]);
            if (m < 8) s[m] = fma(wb * pw, CS[m], s[m]);
            pw *= u2;
        }
    }
    double cs17[17];
#pragma unroll
    for (int m = 0; m < 9; ++m) cs17[m] = c[m];
#pragma unroll
    for (int m = 0; m < 8; ++m) cs17[9 + m] = s[m];
    tm.sumv(cs17);                  // the 17 moments in one reduction
    if (threadIdx.x == 0)
#pragma unroll
        for (int m = 0; m < 17; ++m) mom[m] = cs17[m];
    cg::this_cluster().sync();      // peers are done reading this CTA's slots; mom[] visible
    if (rank != 0) return;          // the grid search and the writes are rank 0's
    double bv = -1.0, hv = 0.0;
    int bi = -1;
    for (int g = threadIdx.x; g < a.n_grid; g += POLISH_THREADS) {
        const double z = a.grid[g] * 1.0e4, z2 = z * z;
        double hc = 0.0, hs = 0.0, pw = 1.0;
#pragma unroll
        for (int m = 0; m < 9; ++m) {
            hc = fma(mom[m], pw, hc);
            if (m < 8) hs = fma(mom[9 + m], pw * z, hs);
            pw *= z2;
        }
        const double h = hc - hs;
        if (fabs(h) > bv) {
            bv = fabs(h);
            bi = g;
            hv = h;
        }
    }
    best_v[threadIdx.x] = bv;
    best_i[threadIdx.x] = bi;
    best_h[threadIdx.x] = hv;
    __syncthreads();
    // first index of the largest |h|: ties go to the smaller grid index
    for (int o = POLISH_THREADS / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            const double v2 = best_v[threadIdx.x + o];
            const int i2 = best_i[threadIdx.x + o];
            if (i2 >= 0 && (v2 > best_v[threadIdx.x] || (v2 == best_v[threadIdx.x] && i2 < best_i[threadIdx.x]) ||
                            best_i[threadIdx.x] < 0)) {
                best_v[threadIdx.x] = v2;
                best_i[threadIdx.x] = i2;
                best_h[threadIdx.x] = best_h[threadIdx.x + o];
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        a.h_unpol[p] = mom[0];
        const int g = best_i[0];
        a.ddy_pol[p] = g >= 0 ? a.grid[g] : 0.0;
        a.h_pol[p] = g >= 0 ? best_h[0] : mom[0];
    }
}

}  // namespace mb
