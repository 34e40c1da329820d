// Exact phase export and the plain FP64 K2 kernel (value + dK2/ddelta + dK2/dk).
//
// Plain method: the phase frac(v G) is reduced exactly with 32x32->64 integer multiplies
// on 32-bit limbs (search/path1_eval_fast.cpp:41-46 does the same product with u128),
// sine/cosine in FP64 from the half-angle polynomials, FP64 accumulation, warp-shuffle
// reduction inside the CTA and a deterministic FP64 reduction across zero chunks.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "k2_common.cuh"
#include "k2_internal.h"

namespace mb {

// ------------------------------------------------------------------ phase export

__global__ void phase128_kernel(TabView t, CandView c, int64_t n_zeros, uint64_t *out_hi,
                                uint64_t *out_lo) {
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t total = c.P * n_zeros;
    if (idx >= total) return;
    int64_t p = idx / n_zeros, j = idx - p * n_zeros;
    Cand64 v = fold_delta(c.vi[p], c.vf[p], c.delta ? c.delta[p] : 0.0);
    uint64_t hi, lo;
    phase128_exact((uint32_t)v.vf, (uint32_t)(v.vf >> 32), (uint32_t)v.vi, (uint32_t)(v.vi >> 32),
                   t.g0[j], t.g1[j], t.g2[j], t.g3[j], t.g4[j], hi, lo);
    out_hi[idx] = hi;
    out_lo[idx] = lo;
}

int launch_phase128(const Table &t, CandView c, int64_t n_zeros, uint64_t *d_hi, uint64_t *d_lo,
                    cudaStream_t s) {
    int64_t total = c.P * n_zeros;
    if (total == 0) return MB_OK;
    int64_t blocks = (total + 255) / 256;
    phase128_kernel<<<(unsigned)blocks, 256, 0, s>>>(view(t), c, n_zeros, d_hi, d_lo);
    MB_CUDA(cudaGetLastError());
    return MB_OK;
}

// ------------------------------------------------------------------ plain K2

constexpr int PLAIN_THREADS = 256;
constexpr int PLAIN_TILE = 256;   // zeros staged per shared-memory tile

struct __align__(16) ZRecPlain {
    uint32_t g0, g1, g2, g3;
    uint32_t g4, pad0, pad1, pad2;
    double wcr, wci, gam, gam2;   // w Re c, w Im c, gamma, gamma^2 with w = exp(-k gamma^2)
};

// Launch shape of the plain kernel: CPT candidates per thread; each candidate's zeros are
// split over LPC lanes of one warp (LPC | 32) and over NZW warps.
struct PlainShape {
    int cpt, lpc_log2, nzw;
    int cands_per_cta() const { return (PLAIN_THREADS / 32 / nzw) * (32 >> lpc_log2) * cpt; }
};

// sin/cos(2 pi hi 2^-64) of the exact 64-bit phase word: the nearest of PLAIN_TAB table angles
// (the top 11 bits of hi + 2^52) and the remainder r = ((hi + 2^52) mod 2^53 - 2^52) 2^-64 turn,
// exact in FP64 (|r| <= 2^-12), rotated by
//   cos(2 pi r) - 1 = r^2 (-2 pi^2 + r^2 2 pi^4 / 3)     (truncation 1.8e-20)
//   sin(2 pi r)     = r (2 pi - r^2 4 pi^3 / 3)           (truncation 7.1e-17)
// so the result is within ~4e-16 of the exact values (table entries rounded once, four FMA
// roundings).  11 FP64 operations and one shared-memory load instead of a 21-operation
// polynomial pair on the full turn.
constexpr int PLAIN_TAB = 2048;
MB_DEV void sincos_phase64_tab(uint64_t hi, const double2 *tab, double &sn, double &cs) {
    const uint64_t h = hi + (1ull << 52);
    const int q = (int)(h >> 53);
    const int32_t rh = (int32_t)((uint32_t)(h >> 32) & 0x1FFFFFu) - (1 << 20);
    const double r = fma(s32_to_f64(rh), 2.3283064365386963e-10, u32_to_f64((uint32_t)h) * 5.421010862427522e-20);
    const double u = r * r;
    const double s = r * fma(u, -41.341702240399755, 6.283185307179586);
    const double cm1 = u * fma(u, 64.93939402266829, -19.739208802178716);
    const double2 T = tab[q];
    cs = fma(T.x, cm1, fma(-T.y, s, T.x));
    sn = fma(T.y, cm1, fma(T.x, s, T.y));
}

template <int CPT>
__global__ void __launch_bounds__(PLAIN_THREADS)
k2_plain_kernel(TabView t, CandView c, int64_t n_use, int64_t chunk, double k, int lpc_log2,
                int nzw, double *partial) {
    __shared__ ZRecPlain tile[PLAIN_TILE];
    __shared__ double2 s_tab[PLAIN_TAB];       // (cos, sin)(2 pi i / PLAIN_TAB); the first tile's
    for (int i = threadIdx.x; i < PLAIN_TAB; i += PLAIN_THREADS) {   // barrier publishes it
        double sn, cs;
        sincospi((double)i * (2.0 / PLAIN_TAB), &sn, &cs);
        s_tab[i] = make_double2(cs, sn);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int lpc = 1 << lpc_log2;
    const int cgroup = warp / nzw, zw = warp - cgroup * nzw;
    const int clane = lane >> lpc_log2, zl_in = lane & (lpc - 1);
    const int ZL = nzw << lpc_log2, zl = zw * lpc + zl_in;
    const int cands_per_warp = 32 >> lpc_log2;
    const int cands_per_cta = (PLAIN_THREADS / 32 / nzw) * cands_per_warp * CPT;
    const int64_t cbase = (int64_t)blockIdx.x * cands_per_cta + (int64_t)(cgroup * cands_per_warp + clane) * CPT;

    uint32_t v0[CPT], v1[CPT], v2[CPT], v3[CPT];
    double sv[CPT], sd[CPT], sk[CPT];
#pragma unroll
    for (int i = 0; i < CPT; ++i) {
        int64_t p = cbase + i;
        Cand64 v{0, 0};
        if (p < c.P) v = fold_delta(c.vi[p], c.vf[p], c.delta ? c.delta[p] : 0.0);
        v0[i] = (uint32_t)v.vf;
        v1[i] = (uint32_t)(v.vf >> 32);
        v2[i] = (uint32_t)v.vi;
        v3[i] = (uint32_t)(v.vi >> 32);
        sv[i] = sd[i] = sk[i] = 0.0;
    }

    const int64_t z0 = (int64_t)blockIdx.y * chunk;
    const int64_t z1 = min(z0 + chunk, n_use);
    for (int64_t tb = z0; tb < z1; tb += PLAIN_TILE) {
        __syncthreads();
        int64_t j = tb + threadIdx.x;
        if (threadIdx.x < PLAIN_TILE && j < z1) {
            double g = t.gamma[j];
            double w = exp(-k * g * g);
            ZRecPlain r;
            r.g0 = t.g0[j]; r.g1 = t.g1[j]; r.g2 = t.g2[j]; r.g3 = t.g3[j]; r.g4 = t.g4[j];
            r.pad0 = r.pad1 = r.pad2 = 0;
            r.wcr = w * t.cre[j];
            r.wci = w * t.cim[j];
            r.gam = g;
            r.gam2 = g * g;
            tile[threadIdx.x] = r;
        }
        __syncthreads();
        const int nt = (int)min((int64_t)PLAIN_TILE, z1 - tb);
        for (int jj = zl; jj < nt; jj += ZL) {
            const ZRecPlain r = tile[jj];
#pragma unroll
            for (int i = 0; i < CPT; ++i) {
                uint64_t hi, lo;
                phase128_exact(v0[i], v1[i], v2[i], v3[i], r.g0, r.g1, r.g2, r.g3, r.g4, hi, lo);
                double s, co;
                sincos_phase64_tab(hi, s_tab, s, co);
                double wre = fma(r.wcr, co, -r.wci * s);
                double wim = fma(r.wcr, s, r.wci * co);
                sv[i] += wre;
                sd[i] = fma(r.gam, wim, sd[i]);
                sk[i] = fma(r.gam2, wre, sk[i]);
            }
        }
    }

    // reduce over the LPC lanes of each candidate
#pragma unroll
    for (int i = 0; i < CPT; ++i) {
        sv[i] = warp_sum_xor(sv[i], lpc);
        sd[i] = warp_sum_xor(sd[i], lpc);
        sk[i] = warp_sum_xor(sk[i], lpc);
    }
    // reduce over the NZW warps of each candidate group (through shared memory)
    __syncthreads();
    double *red = reinterpret_cast<double *>(tile);   // 8 warps * 32 lanes * CPT * 3 doubles
    if (nzw > 1) {
        if (zl_in == 0) {
#pragma unroll
            for (int i = 0; i < CPT; ++i) {
                double *d = red + ((warp * 32 + clane) * CPT + i) * 3;
                d[0] = sv[i]; d[1] = sd[i]; d[2] = sk[i];
            }
        }
        __syncthreads();
        if (zw == 0 && zl_in == 0) {
            for (int w2 = 1; w2 < nzw; ++w2) {
#pragma unroll
                for (int i = 0; i < CPT; ++i) {
                    const double *d = red + (((warp + w2) * 32 + clane) * CPT + i) * 3;
                    sv[i] += d[0]; sd[i] += d[1]; sk[i] += d[2];
                }
            }
        }
    }
    if (zw == 0 && zl_in == 0) {
#pragma unroll
        for (int i = 0; i < CPT; ++i) {
            int64_t p = cbase + i;
            if (p < c.P) {
                double *o = partial + ((int64_t)blockIdx.y * c.P + p) * 3;
                o[0] = sv[i]; o[1] = sd[i]; o[2] = sk[i];
            }
        }
    }
}

// Sum the per-chunk partials in chunk order (deterministic) and apply the factors 2, -2, -2.
__global__ void reduce_partials_kernel(const double *partial, int64_t P, int n_chunk, double *val,
                                       double *dd, double *dk) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    double a = 0, b = 0, e = 0;
    for (int ch = 0; ch < n_chunk; ++ch) {
        const double *o = partial + ((int64_t)ch * P + p) * 3;
        a += o[0]; b += o[1]; e += o[2];
    }
    if (val) val[p] = 2.0 * a;
    if (dd) dd[p] = -2.0 * b;
    if (dk) dk[p] = -2.0 * e;
}

static PlainShape plain_shape(int64_t P) {
    if (P >= 2048) return {2, 0, 1};
    if (P >= 256) return {1, 0, 1};
    if (P >= 64) return {1, 2, 1};
    if (P >= 8) return {1, 5, 1};
    return {1, 5, 8};
}

static int sm_count(int device) {
    static int cached[64] = {0};
    if (device >= 0 && device < 64 && cached[device]) return cached[device];
    int n = 148;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
    if (device >= 0 && device < 64) cached[device] = n;
    return n;
}

// The current context handle through the driver's cuCtxGetCurrent (fetched with
// cudaGetDriverEntryPoint, so the library does not link the driver library itself); null if it
// cannot be had.
void *current_context() {
    typedef int (*ctx_fn)(void **);
    static ctx_fn fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return (ctx_fn)f;
    }();
    void *ctx = nullptr;
    if (fn && fn(&ctx) != 0) ctx = nullptr;
    return ctx;
}

// The plain kernel holds 48 KB of static shared memory (tile + sine/cosine table): ask for the
// largest shared-memory carveout so four CTAs fit on an SM.  Once per device and context.
static int plain_kernel_attributes(int device) {
    static void *done_ctx[64] = {};             // the context the attributes were set in
    void *ctx = current_context();
    if (device >= 0 && device < 64 && ctx && done_ctx[device] == ctx) return MB_OK;
    MB_CUDA(cudaFuncSetAttribute(k2_plain_kernel<1>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared));
    MB_CUDA(cudaFuncSetAttribute(k2_plain_kernel<2>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared));
    if (device >= 0 && device < 64) done_ctx[device] = current_context();
    return MB_OK;
}

int launch_plain(Table &t, CandView c, int64_t n_use, double k, double *d_val, double *d_dd,
                 double *d_dk, cudaStream_t s, double *d_partial_override, size_t partial_cap) {
    if (c.P == 0) return MB_OK;
    MB_TRY(plain_kernel_attributes(t.device));
    PlainShape sh = plain_shape(c.P);
    int64_t cta_c = sh.cands_per_cta();
    int64_t n_ctile = (c.P + cta_c - 1) / cta_c;
    int64_t target = (int64_t)sm_count(t.device) * 8;          // ~4 waves of 2 CTAs/SM
    int64_t n_chunk = std::max<int64_t>(1, (target + n_ctile - 1) / n_ctile);
    int64_t max_chunks = std::max<int64_t>(1, (n_use + PLAIN_TILE - 1) / PLAIN_TILE);
    n_chunk = std::min(n_chunk, max_chunks);
    int64_t chunk = (n_use + n_chunk - 1) / n_chunk;
    chunk = ((chunk + PLAIN_TILE - 1) / PLAIN_TILE) * PLAIN_TILE;
    if (chunk == 0) chunk = PLAIN_TILE;
    n_chunk = std::max<int64_t>(1, (n_use + chunk - 1) / chunk);
    size_t need = (size_t)n_chunk * c.P * 3 * sizeof(double);
    double *partial = d_partial_override;
    if (partial) {
        if (need > partial_cap) {
            set_error("plain: partial buffer needs %zu bytes, have %zu", need, partial_cap);
            return MB_ERR_CAPACITY;
        }
    } else {
        MB_TRY(t.work.ensure(need));
        partial = (double *)t.work.p;
    }
    if (n_use == 0) {
        MB_CUDA(cudaMemsetAsync(partial, 0, (size_t)c.P * 3 * sizeof(double), s));
        n_chunk = 1;
    } else {
        dim3 grid((unsigned)n_ctile, (unsigned)n_chunk);
        if (sh.cpt == 2)
            k2_plain_kernel<2><<<grid, PLAIN_THREADS, 0, s>>>(view(t), c, n_use, chunk, k, sh.lpc_log2, sh.nzw, partial);
        else
            k2_plain_kernel<1><<<grid, PLAIN_THREADS, 0, s>>>(view(t), c, n_use, chunk, k, sh.lpc_log2, sh.nzw, partial);
        MB_CUDA(cudaGetLastError());
    }
    reduce_partials_kernel<<<(unsigned)((c.P + 255) / 256), 256, 0, s>>>(partial, c.P, (int)n_chunk, d_val, d_dd, d_dk);
    MB_CUDA(cudaGetLastError());
    return MB_OK;
}

}  // namespace mb

// ------------------------------------------------------------------ no-allocation entry point
//
// For callers that cannot allocate device memory themselves: code running where cudaMalloc is
// not allowed or not wanted (inside a host callback, a real-time or pre-reserved memory budget,
// an embedding runtime that owns all allocations).  The per-chunk partial sums of the plain
// kernel go to a fixed file-scope device array instead of a table-owned buffer, and the zero
// data and candidates are passed as plain device pointers, so a call allocates nothing.
//
// The array holds NOALLOC_PARTIAL_DOUBLES doubles (8 MiB); every GPU that loads this library
// keeps it until the process exits.  P is limited to NOALLOC_PARTIAL_DOUBLES / 3 candidates.
// All calls on a device share the array: calls that overlap on the GPU (different streams,
// host threads) race on it.  A call overwrites every slot it later reads, so no earlier
// contents leak into a result.  The first call on a device looks up the array's device
// address (cudaGetSymbolAddress); make that first call before any stream capture.  The address
// is kept with the device's current context and looked up again when the context changes (after
// a cudaDeviceReset the array lives at a new address in the new primary context).
namespace {

constexpr int64_t NOALLOC_PARTIAL_DOUBLES = (int64_t)1 << 20;
static __device__ __align__(256) double g_noalloc_partial[NOALLOC_PARTIAL_DOUBLES];

constexpr int NOALLOC_MAX_DEVICES = 64;
double *g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};
void *g_noalloc_ctx[NOALLOC_MAX_DEVICES] = {};
std::mutex g_noalloc_mu;

// Device address of the array on the current device (set up once per device and context).
int noalloc_scratch(double **out) {
    int dev = -1;
    MB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        mb::set_error("no-allocation scratch: device %d out of range", dev);
        return MB_ERR_ARG;
    }
    void *ctx = mb::current_context();
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev] || ctx != g_noalloc_ctx[dev]) {
        double *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_partial);
        if (e != cudaSuccess || p == nullptr) {
            mb::set_error("cudaGetSymbolAddress for the no-allocation scratch failed: %s",
                          cudaGetErrorString(e));
            return MB_ERR_CUDA;
        }
        g_noalloc_addr[dev] = p;
        g_noalloc_ctx[dev] = mb::current_context();     // current now, if it was not on entry
    }
    *out = g_noalloc_addr[dev];
    return MB_OK;
}

}  // namespace

extern "C" int mb_k2_plain_noalloc_dev(const uint32_t *d_g, const double *d_gamma, const double *d_cre,
                                       const double *d_cim, int64_t n_zeros, int64_t n_use, int64_t P,
                                       const uint64_t *d_v_int, const uint64_t *d_v_frac,
                                       const double *d_delta, double k, double *d_val, double *d_dd,
                                       double *d_dk, void *stream) {
    using namespace mb;
    MB_CHECK_ARG(P >= 0, "mb_k2_plain_noalloc_dev: P=%lld", (long long)P);
    if (P * 3 > NOALLOC_PARTIAL_DOUBLES) {
        set_error("mb_k2_plain_noalloc_dev: P=%lld exceeds the fixed scratch (at most %lld candidates)",
                  (long long)P, (long long)(NOALLOC_PARTIAL_DOUBLES / 3));
        return MB_ERR_CAPACITY;
    }
    MB_CHECK_ARG(d_g && d_gamma && d_cre && d_cim && d_v_int && d_v_frac && d_val && d_dd && d_dk,
                 "mb_k2_plain_noalloc_dev: null argument");
    MB_CHECK_ARG(n_zeros >= 1 && n_use >= 0 && n_use <= n_zeros, "mb_k2_plain_noalloc_dev: n_use=%lld n_zeros=%lld",
                 (long long)n_use, (long long)n_zeros);
    MB_CHECK_ARG(std::isfinite(k) && k >= 0.0, "mb_k2_plain_noalloc_dev: k=%g", k);
    if (P == 0) return MB_OK;
    double *partial = nullptr;
    MB_TRY(noalloc_scratch(&partial));
    int dev = 0;
    MB_CUDA(cudaGetDevice(&dev));
    cudaStream_t s = (cudaStream_t)stream;
    TabView tv{};
    tv.g0 = d_g;
    tv.g1 = d_g + n_zeros;
    tv.g2 = d_g + 2 * n_zeros;
    tv.g3 = d_g + 3 * n_zeros;
    tv.g4 = d_g + 4 * n_zeros;
    tv.gamma = d_gamma;
    tv.cre = d_cre;
    tv.cim = d_cim;
    tv.n = n_zeros;
    CandView c{d_v_int, d_v_frac, d_delta, P};
    MB_TRY(plain_kernel_attributes(dev));
    PlainShape sh = plain_shape(P);
    int64_t cta_c = sh.cands_per_cta();
    int64_t n_ctile = (P + cta_c - 1) / cta_c;
    int64_t n_chunk = std::max<int64_t>(1, ((int64_t)sm_count(dev) * 8 + n_ctile - 1) / n_ctile);
    n_chunk = std::min(n_chunk, std::max<int64_t>(1, (n_use + PLAIN_TILE - 1) / PLAIN_TILE));
    n_chunk = std::min(n_chunk, NOALLOC_PARTIAL_DOUBLES / (3 * P));      // fits the fixed array
    int64_t chunk = std::max<int64_t>(1, (n_use + n_chunk - 1) / n_chunk);
    chunk = ((chunk + PLAIN_TILE - 1) / PLAIN_TILE) * PLAIN_TILE;
    n_chunk = std::max<int64_t>(1, (n_use + chunk - 1) / chunk);
    if (n_use == 0) {
        // nothing to sum: clear the one chunk the reduction reads
        MB_CUDA(cudaMemsetAsync(partial, 0, (size_t)P * 3 * sizeof(double), s));
        n_chunk = 1;
    } else {
        dim3 grid((unsigned)n_ctile, (unsigned)n_chunk);
        if (sh.cpt == 2)
            k2_plain_kernel<2><<<grid, PLAIN_THREADS, 0, s>>>(tv, c, n_use, chunk, k, sh.lpc_log2, sh.nzw, partial);
        else
            k2_plain_kernel<1><<<grid, PLAIN_THREADS, 0, s>>>(tv, c, n_use, chunk, k, sh.lpc_log2, sh.nzw, partial);
        MB_CUDA(cudaGetLastError());
    }
    reduce_partials_kernel<<<(unsigned)((P + 255) / 256), 256, 0, s>>>(partial, P, (int)n_chunk, d_val, d_dd, d_dk);
    MB_CUDA(cudaGetLastError());
    return MB_OK;
}
