// Zero-table creation, validation and lifetime; error-state plumbing.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstring>

#include "k2_internal.h"

struct mb_table {
    mb::Table t;
};

namespace mb {

static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

const char *last_error() { return g_err; }

int device_guard(int device) {
    int cur = -1;
    MB_CUDA(cudaGetDevice(&cur));
    if (cur != device) MB_CUDA(cudaSetDevice(device));
    return MB_OK;
}

int64_t Table::count_below(double T) const {
    if (!(T < INFINITY)) return n;
    return (int64_t)(std::lower_bound(h_gamma.begin(), h_gamma.end(), T) - h_gamma.begin());
}

int DevBuf::ensure(size_t need) {
    if (need <= bytes) return MB_OK;
    if (p) {
        MB_CUDA(cudaDeviceSynchronize());
        MB_CUDA(cudaFree(p));
        p = nullptr;
        bytes = 0;
    }
    size_t want = std::max(need + need / 4, (size_t)1 << 20);
    MB_CUDA(cudaMalloc(&p, want));
    bytes = want;
    return MB_OK;
}

void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

TabView view(const Table &t) {
    TabView v;
    v.g0 = t.d_g;
    v.g1 = t.d_g + t.n;
    v.g2 = t.d_g + 2 * t.n;
    v.g3 = t.d_g + 3 * t.n;
    v.g4 = t.d_g + 4 * t.n;
    v.gamma = t.d_gamma;
    v.cre = t.d_cre;
    v.cim = t.d_cim;
    v.alpha = t.d_alpha;
    v.psi = t.d_psi;
    v.n = t.n;
    return v;
}

static void free_table(Table &t) {
    cudaFree(t.d_g);
    cudaFree(t.d_gamma);
    cudaFree(t.d_cre);
    cudaFree(t.d_cim);
    cudaFree(t.d_alpha);
    cudaFree(t.d_psi);
    t.io.release();
    t.work.release();
    t.screen.release();
    for (double *w : t.d_weights) cudaFree(w);
    if (t.ev_fork) cudaEventDestroy(t.ev_fork);
    if (t.ev_join) cudaEventDestroy(t.ev_join);
    if (t.side) cudaStreamDestroy(t.side);
    if (t.stream) cudaStreamDestroy(t.stream);
    t = Table();
}

}  // namespace mb

using namespace mb;

extern "C" const char *mb_last_error(void) { return mb::last_error(); }

extern "C" int mb_abi_version(void) { return 1; }

extern "C" int mb_table_create(const uint64_t *G3, const double *c_re, const double *c_im,
                               const double *gamma, int64_t n, int device, mb_table **out) {
    MB_CHECK_ARG(out != nullptr, "mb_table_create: out is null");
    *out = nullptr;
    MB_CHECK_ARG(G3 && c_re && c_im && gamma, "mb_table_create: null array");
    MB_CHECK_ARG(n >= 1 && n <= ((int64_t)1 << 31), "mb_table_create: n=%lld out of range",
                 (long long)n);
    MB_CHECK_ARG(device >= 0, "mb_table_create: device %d", device);

    // ---- validation (host, O(n)), before any CUDA call
    const long double two_pi = 6.28318530717958647692528676655900577L;
    for (int64_t j = 0; j < n; ++j) {
        double g = gamma[j];
        if (!(std::isfinite(g) && g > 0.0)) {
            set_error("mb_table_create: gamma[%lld]=%g is not finite and positive", (long long)j, g);
            return MB_ERR_TABLE;
        }
        if (j > 0 && !(g > gamma[j - 1])) {
            set_error("mb_table_create: gamma not strictly increasing at %lld", (long long)j);
            return MB_ERR_TABLE;
        }
        if (!(std::isfinite(c_re[j]) && std::isfinite(c_im[j]))) {
            set_error("mb_table_create: non-finite c at %lld", (long long)j);
            return MB_ERR_TABLE;
        }
        if (G3[3 * j] >> 32) {
            set_error("mb_table_create: G integer part >= 2^32 at %lld", (long long)j);
            return MB_ERR_TABLE;
        }
        long double G = (long double)G3[3 * j] + ldexpl((long double)G3[3 * j + 1], -64) +
                        ldexpl((long double)G3[3 * j + 2], -128);
        long double diff = fabsl(two_pi * G - (long double)g);
        if (diff > 4.0L * (long double)(nextafter(g, INFINITY) - g)) {
            set_error("mb_table_create: |gamma - 2pi G| = %Lg exceeds 4 ulp at %lld", diff,
                      (long long)j);
            return MB_ERR_TABLE;
        }
    }

    int ndev = 0;
    MB_CUDA(cudaGetDeviceCount(&ndev));
    MB_CHECK_ARG(device < ndev, "mb_table_create: device %d of %d", device, ndev);
    MB_TRY(device_guard(device));
    mb_table *h = new mb_table();
    Table &t = h->t;
    t.device = device;
    t.n = n;
    auto fail = [&](int code) {
        free_table(t);
        delete h;
        return code;
    };
    // ---- derived arrays
    std::vector<uint32_t> g(5 * (size_t)n);
    std::vector<uint64_t> psi(n);
    t.h_gamma.assign(gamma, gamma + n);
    t.h_alpha.resize(n);
    for (int64_t j = 0; j < n; ++j) {
        uint64_t gi = G3[3 * j], ghi = G3[3 * j + 1], glo = G3[3 * j + 2];
        g[j] = (uint32_t)glo;
        g[n + j] = (uint32_t)(glo >> 32);
        g[2 * n + j] = (uint32_t)ghi;
        g[3 * n + j] = (uint32_t)(ghi >> 32);
        g[4 * n + j] = (uint32_t)gi;
        t.h_alpha[j] = std::hypot(c_re[j], c_im[j]);
        long double a = atan2l((long double)c_im[j], (long double)c_re[j]) / two_pi;  // (-1/2, 1/2]
        if (a < 0) a += 1.0L;
        long double r = floorl(ldexpl(a, 64) + 0.5L);    // nearest multiple of 2^-64 turn
        psi[j] = (r >= 18446744073709551616.0L) ? 0 : (uint64_t)r;
    }
    cudaError_t e;
#define ALLOC_COPY(dst, src, bytes)                                                    \
    if ((e = cudaMalloc((void **)&dst, bytes)) != cudaSuccess ||                       \
        (e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice)) != cudaSuccess) {    \
        set_error("mb_table_create: %s", cudaGetErrorString(e));                       \
        return fail(MB_ERR_CUDA);                                                      \
    }
    ALLOC_COPY(t.d_g, g.data(), 5 * (size_t)n * sizeof(uint32_t));
    ALLOC_COPY(t.d_gamma, gamma, n * sizeof(double));
    ALLOC_COPY(t.d_cre, c_re, n * sizeof(double));
    ALLOC_COPY(t.d_cim, c_im, n * sizeof(double));
    ALLOC_COPY(t.d_alpha, t.h_alpha.data(), n * sizeof(double));
    ALLOC_COPY(t.d_psi, psi.data(), n * sizeof(uint64_t));
#undef ALLOC_COPY
    if ((e = cudaStreamCreateWithFlags(&t.stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&t.side, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&t.ev_fork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&t.ev_join, cudaEventDisableTiming)) != cudaSuccess) {
        set_error("mb_table_create: %s", cudaGetErrorString(e));
        return fail(MB_ERR_CUDA);
    }
    *out = h;
    return MB_OK;
}

extern "C" int mb_table_destroy(mb_table *h) {
    if (!h) return MB_OK;
    if (h->t.n_plans > 0) {
        set_error("mb_table_destroy: %d plan(s) still use this table; destroy them first", h->t.n_plans);
        return MB_ERR_STATE;
    }
    device_guard(h->t.device);
    free_table(h->t);
    delete h;
    return MB_OK;
}

extern "C" int mb_table_size(const mb_table *h, int64_t *n_out) {
    MB_CHECK_ARG(h && n_out, "mb_table_size: null argument");
    *n_out = h->t.n;
    return MB_OK;
}

extern "C" int mb_table_count_below(const mb_table *h, double T, int64_t *n_out) {
    MB_CHECK_ARG(h && n_out, "mb_table_count_below: null argument");
    MB_CHECK_ARG(!std::isnan(T), "mb_table_count_below: T is NaN");
    *n_out = h->t.count_below(T);
    return MB_OK;
}

extern "C" int mb_table_add_weights(mb_table *h, const double *w, int64_t n, int *slot) {
    MB_CHECK_ARG(h && w && slot, "mb_table_add_weights: null argument");
    Table &t = h->t;
    MB_CHECK_ARG(n == t.n, "mb_table_add_weights: %lld weights for a table of %lld zeros", (long long)n,
                 (long long)t.n);
    MB_CHECK_ARG(t.d_weights.size() < 64, "mb_table_add_weights: at most 64 weight vectors per table");
    for (int64_t j = 0; j < n; ++j)
        if (!std::isfinite(w[j])) {
            set_error("mb_table_add_weights: weight %lld is not finite", (long long)j);
            return MB_ERR_TABLE;
        }
    MB_TRY(device_guard(t.device));
    double *d = nullptr;
    MB_CUDA(cudaMalloc(&d, n * sizeof(double)));
    cudaError_t e = cudaMemcpy(d, w, n * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        set_error("mb_table_add_weights: %s", cudaGetErrorString(e));
        return MB_ERR_CUDA;
    }
    t.d_weights.push_back(d);
    t.h_weights.emplace_back(w, w + n);
    *slot = (int)t.d_weights.size() - 1;
    return MB_OK;
}

// Accessor used by the other translation units.
namespace mb {
Table &table_of(mb_table *h) { return h->t; }
}  // namespace mb
