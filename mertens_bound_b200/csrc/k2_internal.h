// Host-side internals of libmertens_k2.so (not part of the public C-ABI).
#pragma once
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/mertens_k2.h"

namespace mb {

// Thread-local last-error message (mb_last_error()).
void set_error(const char *fmt, ...);
// The calling thread's current CUDA context (the driver's cuCtxGetCurrent), or null: per-device
// caches key on it, so they are refreshed after a context is replaced (cudaDeviceReset).
void *current_context();
const char *last_error();

// Return-on-error helpers used by every entry point.
#define MB_CHECK_ARG(cond, ...)                          \
    do {                                                 \
        if (!(cond)) {                                   \
            ::mb::set_error(__VA_ARGS__);                \
            return MB_ERR_ARG;                           \
        }                                                \
    } while (0)

#define MB_CUDA(call)                                                                       \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            ::mb::set_error("CUDA error %s (%s) at %s:%d", cudaGetErrorName(e_),            \
                            cudaGetErrorString(e_), __FILE__, __LINE__);                    \
            return MB_ERR_CUDA;                                                             \
        }                                                                                   \
    } while (0)

#define MB_TRY(call)              \
    do {                          \
        int s_ = (call);          \
        if (s_ != MB_OK) return s_; \
    } while (0)

// Grow-only device buffer.  ensure() synchronises the device before it frees a smaller
// buffer, so work still in flight on any stream never sees its memory released.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    int ensure(size_t need);
    void release();
};

// Device-resident zero table.  Planar (structure of arrays), every array 256-byte aligned:
//   g[0..4][n]  u32 limbs of G 2^128 (g0 least significant .. g4 = integer part)
//   gamma[n], c_re[n], c_im[n]    FP64 as given
//   alpha[n] = |c|, psi[n] = round(frac(arg(c)/2pi) 2^64)   (derived at creation)
struct Table {
    int device = 0;
    int64_t n = 0;
    uint32_t *d_g = nullptr;          // 5*n words, limb-major
    double *d_gamma = nullptr, *d_cre = nullptr, *d_cim = nullptr;
    double *d_alpha = nullptr;
    uint64_t *d_psi = nullptr;
    std::vector<double> h_gamma;      // host copies for cutoffs and error planning
    std::vector<double> h_alpha;
    // per-zero weight vectors registered with the table (device copies + host copies)
    std::vector<double *> d_weights;
    std::vector<std::vector<double>> h_weights;
    cudaStream_t stream = nullptr;    // the library's own stream for host-pointer calls
    cudaStream_t side = nullptr;      // second stream: heavy tier beside the light tier
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // grow-only scratch owned by the table: `io` stages candidates and results of host-pointer
    // calls, `work` holds per-chunk partial sums, `screen` the zero records of mb_screen_dev
    // (which runs on the caller's stream, so it shares no buffer with calls on `stream`).  Calls
    // on one table that use the same buffer must not overlap on the GPU.
    DevBuf io, work, screen;
    int n_plans = 0;                  // live plans on this table (it cannot be destroyed under them)

    int64_t count_below(double T) const;
};

// Device view of the table passed to kernels by value.
struct TabView {
    const uint32_t *g0, *g1, *g2, *g3, *g4;
    const double *gamma, *cre, *cim, *alpha;
    const uint64_t *psi;
    int64_t n;
};

TabView view(const Table &t);

// Candidate arrays on the device.
struct CandView {
    const uint64_t *vi, *vf;
    const double *delta;   // may be null (all zero)
    int64_t P;
};

int device_guard(int device);

// Per-device grow-only scratch of the handle-free entry points (reference-compatible calls);
// hold scratch_mutex() while using it.
std::mutex &scratch_mutex();
int scratch_buffer(size_t bytes, void **out);

// Bump allocation of 256-byte aligned sub-arrays from a scratch block.
template <typename T>
T *carve(char *&p, size_t n) {
    T *r = (T *)p;
    p += ((n * sizeof(T) + 255) / 256) * 256;
    return r;
}

// Kernel launchers (return MB_OK or an MB_ERR_* code).
Table &table_of(struct ::mb_table *h);

int launch_phase128(const Table &t, CandView c, int64_t n_zeros, uint64_t *d_hi, uint64_t *d_lo,
                    cudaStream_t s);
int launch_plain(Table &t, CandView c, int64_t n_use, double k, double *d_val, double *d_dd,
                 double *d_dk, cudaStream_t s, double *d_partial_override = nullptr,
                 size_t partial_cap = 0);

}  // namespace mb
