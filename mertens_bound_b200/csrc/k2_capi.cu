// C-ABI entry points: argument checks, host<->device staging, kernel dispatch.
#include <cmath>
#include <cstring>

#include "k2_internal.h"

using namespace mb;

namespace {

// Host-pointer candidates staged into the table's `io` buffer; layout:
//   vi[P] | vf[P] | delta[P] | out (n_out_words u64/f64)
struct Staged {
    uint64_t *vi, *vf;
    double *delta;
    void *out;
};

int stage_candidates(Table &t, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                     const double *delta, size_t out_bytes, Staged &s) {
    size_t cand = (size_t)P * 8;
    size_t need = 3 * cand + out_bytes + 256;
    MB_TRY(t.io.ensure(need));
    char *base = (char *)t.io.p;
    s.vi = (uint64_t *)base;
    s.vf = (uint64_t *)(base + cand);
    s.delta = (double *)(base + 2 * cand);
    s.out = (void *)(base + ((3 * cand + 255) & ~(size_t)255));
    MB_CUDA(cudaMemcpyAsync(s.vi, v_int, cand, cudaMemcpyHostToDevice, t.stream));
    MB_CUDA(cudaMemcpyAsync(s.vf, v_frac, cand, cudaMemcpyHostToDevice, t.stream));
    if (delta)
        MB_CUDA(cudaMemcpyAsync(s.delta, delta, cand, cudaMemcpyHostToDevice, t.stream));
    else
        MB_CUDA(cudaMemsetAsync(s.delta, 0, cand, t.stream));
    return MB_OK;
}

int check_k_T(double k, double T, const char *who) {
    MB_CHECK_ARG(std::isfinite(k) && k >= 0.0, "%s: k=%g must be finite and >= 0", who, k);
    MB_CHECK_ARG(!std::isnan(T), "%s: T is NaN", who);
    return MB_OK;
}

int check_delta_host(int64_t P, const double *delta, const char *who) {
    if (!delta) return MB_OK;
    for (int64_t p = 0; p < P; ++p)
        MB_CHECK_ARG(std::isfinite(delta[p]) && std::fabs(delta[p]) < 4.0e18,
                     "%s: delta[%lld]=%g is not finite or too large", who, (long long)p, delta[p]);
    return MB_OK;
}

}  // namespace

extern "C" int mb_phase128(mb_table *h, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                           int64_t n_zeros, uint64_t *out_hi, uint64_t *out_lo) {
    MB_CHECK_ARG(h && v_int && v_frac && out_hi && out_lo, "mb_phase128: null argument");
    Table &t = table_of(h);
    MB_CHECK_ARG(P >= 0 && n_zeros >= 0 && n_zeros <= t.n, "mb_phase128: bad sizes P=%lld n=%lld",
                 (long long)P, (long long)n_zeros);
    MB_CHECK_ARG(P * n_zeros <= ((int64_t)1 << 31), "mb_phase128: P*n_zeros too large");
    if (P == 0 || n_zeros == 0) return MB_OK;
    MB_TRY(device_guard(t.device));
    size_t words = (size_t)P * n_zeros;
    Staged s;
    MB_TRY(stage_candidates(t, P, v_int, v_frac, nullptr, 2 * words * 8, s));
    uint64_t *d_hi = (uint64_t *)s.out, *d_lo = d_hi + words;
    MB_TRY(launch_phase128(t, CandView{s.vi, s.vf, s.delta, P}, n_zeros, d_hi, d_lo, t.stream));
    MB_CUDA(cudaMemcpyAsync(out_hi, d_hi, words * 8, cudaMemcpyDeviceToHost, t.stream));
    MB_CUDA(cudaMemcpyAsync(out_lo, d_lo, words * 8, cudaMemcpyDeviceToHost, t.stream));
    MB_CUDA(cudaStreamSynchronize(t.stream));
    return MB_OK;
}

extern "C" int mb_k2_plain(mb_table *h, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                           const double *delta, double k, double T, double *out_val,
                           double *out_dd, double *out_dk) {
    MB_CHECK_ARG(h && v_int && v_frac && out_val, "mb_k2_plain: null argument");
    MB_CHECK_ARG(P >= 0 && P <= ((int64_t)1 << 26), "mb_k2_plain: P=%lld out of range", (long long)P);
    MB_TRY(check_k_T(k, T, "mb_k2_plain"));
    MB_TRY(check_delta_host(P, delta, "mb_k2_plain"));
    if (P == 0) return MB_OK;
    Table &t = table_of(h);
    MB_TRY(device_guard(t.device));
    Staged s;
    MB_TRY(stage_candidates(t, P, v_int, v_frac, delta, 3 * (size_t)P * 8, s));
    double *d_out = (double *)s.out;
    MB_TRY(launch_plain(t, CandView{s.vi, s.vf, s.delta, P}, t.count_below(T), k, d_out, d_out + P,
                        d_out + 2 * P, t.stream));
    MB_CUDA(cudaMemcpyAsync(out_val, d_out, P * 8, cudaMemcpyDeviceToHost, t.stream));
    if (out_dd) MB_CUDA(cudaMemcpyAsync(out_dd, d_out + P, P * 8, cudaMemcpyDeviceToHost, t.stream));
    if (out_dk) MB_CUDA(cudaMemcpyAsync(out_dk, d_out + 2 * P, P * 8, cudaMemcpyDeviceToHost, t.stream));
    MB_CUDA(cudaStreamSynchronize(t.stream));
    return MB_OK;
}

extern "C" int mb_k2_plain_dev(mb_table *h, int64_t P, const uint64_t *d_v_int,
                               const uint64_t *d_v_frac, const double *d_delta, double k, double T,
                               double *d_val, double *d_dd, double *d_dk, void *stream) {
    MB_CHECK_ARG(h && d_v_int && d_v_frac && d_val, "mb_k2_plain_dev: null argument");
    MB_CHECK_ARG(P >= 0 && P <= ((int64_t)1 << 26), "mb_k2_plain_dev: P=%lld out of range", (long long)P);
    MB_TRY(check_k_T(k, T, "mb_k2_plain_dev"));
    if (P == 0) return MB_OK;
    Table &t = table_of(h);
    MB_TRY(device_guard(t.device));
    MB_TRY(launch_plain(t, CandView{d_v_int, d_v_frac, d_delta, P}, t.count_below(T), k, d_val, d_dd,
                        d_dk, (cudaStream_t)stream));
    return MB_OK;
}
