// Leaf screen of the lattice enumerators: a staged K2 proxy at 7 offsets.
//
// Reference: ZeroData::fast_screen (search/fast_mertens_enum.cpp:108-142) and the GPU leaf
// scoring of search/gpu_mertens_stream.cu:192-250.  For a leaf y they sum
//   S_m = sum_j 2|c_j| e^{-3e-9 gamma_j^2} cos(gamma_j (y + m 0.0014) + arg c_j),  m = -3..3,
// over the first 64 zeros, reject the leaf if max_m |S_m| is below a threshold, continue over
// zeros 64..127 (and 128..255 on the GPU) with the next threshold, and report the survivors.
// The reference takes cos from a 4096/16384-entry FP32 table at a phase rounded to 12/14 bits
// and the offset as a rounded table step; here the phase is the 32-bit light-tier phase
// (exact to a few units of 2^-32 turn), cos/sin come from MUFU, the offsets are exact
// (frac(step G) from the 128-bit product), and
//   cos(theta + m D) = cos(theta) cos(m D) - sin(theta) sin(m D)
// gives all 7 offsets from one sin/cos pair per (leaf, zero).  Scores agree with the exact sums
// to ~1e-6 of sum |a|; the reference's table proxy is off by up to ~pi/4096 of sum |a|, so the
// two agree on every leaf not within that distance of a threshold.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "k2_light.cuh"

namespace mb {
namespace {

constexpr int SCREEN_THREADS = 256;
constexpr int SCREEN_MAX_ZEROS = 1024;
constexpr int SCREEN_MAX_STAGES = 8;

struct __align__(16) ZScreen {   // 80 B
    uint32_t b0, b1, gi, psi32;
    double b0s, c1s, gis, b1s;
    float a;                      // 2|c| e^{-k gamma^2}
    float cm[3], sm[3];           // a cos(2 pi m D), a sin(2 pi m D), m = 1..3, D = frac(step G)
    float pad;
};

struct ScreenArgs {
    int n_stages;
    int stage_end[SCREEN_MAX_STAGES];
    float thr[SCREEN_MAX_STAGES];
};

__global__ void screen_prep_kernel(TabView t, int n, double k, uint64_t step_int, uint64_t step_frac, ZScreen *out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    ZScreen r;
    const uint32_t c1 = t.g1[j], b0 = t.g2[j], b1 = t.g3[j], gi = t.g4[j];
    r.b0 = b0;
    r.b1 = b1;
    r.gi = gi;
    r.psi32 = (uint32_t)((t.psi[j] + 0x80000000ull) >> 32) + 2u;
    r.b0s = u32_to_f64(b0) * TWO_M32;
    r.c1s = u32_to_f64(c1) * TWO_M32;
    r.gis = u32_to_f64(gi) * TWO_M32;
    r.b1s = u32_to_f64(b1) * TWO_M32;
    const double g = t.gamma[j];
    const double a = 2.0 * t.alpha[j] * exp(-k * g * g);
    r.a = (float)a;
    uint64_t hi, lo;
    phase128_exact((uint32_t)step_frac, (uint32_t)(step_frac >> 32), (uint32_t)step_int, (uint32_t)(step_int >> 32),
                   t.g0[j], c1, b0, b1, gi, hi, lo);
    const double D = s64_turns_to_f64(hi);      // frac(step G) in [-1/2, 1/2)
#pragma unroll
    for (int m = 1; m <= 3; ++m) {
        double s, c;
        sincospi(2.0 * m * D, &s, &c);
        r.cm[m - 1] = (float)(a * c);
        r.sm[m - 1] = (float)(a * s);
    }
    r.pad = 0.f;
    out[j] = r;
}

__global__ void __launch_bounds__(SCREEN_THREADS) screen_kernel(const ZScreen *zs, int n_zeros, CandView c,
                                                                ScreenArgs sa, int64_t max_hits,
                                                                unsigned long long *count, int64_t *hit_idx,
                                                                float *hit_score, float *scores) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ZScreen *tile = reinterpret_cast<ZScreen *>(smem_raw);
    {
        const int4 *src = reinterpret_cast<const int4 *>(zs);
        int4 *dst = reinterpret_cast<int4 *>(tile);
        const int words = n_zeros * (int)(sizeof(ZScreen) / sizeof(int4));
        for (int i = threadIdx.x; i < words; i += SCREEN_THREADS) dst[i] = src[i];
    }
    __syncthreads();
    const int64_t p = (int64_t)blockIdx.x * SCREEN_THREADS + threadIdx.x;
    const bool valid = p < c.P;
    const CandRegs cr = cand_regs(c, p, valid);
    float S[7];
#pragma unroll
    for (int m = 0; m < 7; ++m) S[m] = 0.f;
    float sc[SCREEN_MAX_STAGES];
    bool alive = valid;
    int reached = 0;
    int j = 0;
    for (int s = 0; s < sa.n_stages; ++s) {
        if (!__any_sync(0xffffffffu, alive)) break;
        const int end = sa.stage_end[s];
        for (; j < end; ++j) {
            const ZScreen z = tile[j];
            const int32_t u = (int32_t)light_phase32(cr, z.b0, z.b1, z.gi, z.b0s, z.c1s, z.gis, z.b1s, z.psi32);
            const float th = (float)u * 1.4629180792671596e-09f;   // 2pi 2^-32
            const float sn = __sinf(th), cs = __cosf(th);
            S[3] = fmaf(z.a, cs, S[3]);
#pragma unroll
            for (int m = 1; m <= 3; ++m) {
                const float x = cs * z.cm[m - 1], y = sn * z.sm[m - 1];
                S[3 + m] += x - y;
                S[3 - m] += x + y;
            }
        }
        float best = 0.f;
#pragma unroll
        for (int m = 0; m < 7; ++m) best = fmaxf(best, fabsf(S[m]));
        sc[s] = best;
        if (alive) reached = s + 1;
        alive = alive && best >= sa.thr[s];
    }
    if (!valid) return;
    if (scores)
        for (int s = 0; s < sa.n_stages; ++s) scores[p * sa.n_stages + s] = s < reached ? sc[s] : -1.0f;
    if (alive && reached == sa.n_stages) {
        const unsigned long long h = atomicAdd(count, 1ull);
        if ((int64_t)h < max_hits) {
            hit_idx[h] = p;
            for (int s = 0; s < sa.n_stages; ++s) hit_score[h * sa.n_stages + s] = sc[s];
        }
    }
}

int screen_args(const Table &t, int n_stages, const int64_t *stage_end, const float *threshold, double k,
                int64_t P, int64_t max_hits, const char *who, ScreenArgs &sa) {
    MB_CHECK_ARG(stage_end && threshold, "%s: null stage argument", who);
    MB_CHECK_ARG(P >= 0 && P <= ((int64_t)1 << 31), "%s: P=%lld", who, (long long)P);
    MB_CHECK_ARG(n_stages >= 1 && n_stages <= SCREEN_MAX_STAGES, "%s: n_stages=%d", who, n_stages);
    MB_CHECK_ARG(std::isfinite(k) && k >= 0, "%s: k=%g", who, k);
    MB_CHECK_ARG(max_hits >= 0, "%s: max_hits=%lld", who, (long long)max_hits);
    sa = ScreenArgs{};
    sa.n_stages = n_stages;
    for (int s = 0; s < n_stages; ++s) {
        MB_CHECK_ARG(stage_end[s] >= 1 && stage_end[s] <= SCREEN_MAX_ZEROS && stage_end[s] <= t.n &&
                         (s == 0 || stage_end[s] > stage_end[s - 1]),
                     "%s: stage_end[%d]=%lld must increase within [1, min(%d, n)]", who, s, (long long)stage_end[s],
                     SCREEN_MAX_ZEROS);
        MB_CHECK_ARG(std::isfinite(threshold[s]), "%s: threshold[%d] is not finite", who, s);
        sa.stage_end[s] = (int)stage_end[s];
        sa.thr[s] = threshold[s];
    }
    return MB_OK;
}

// Zero records into d_z, the count reset, and the screen over P device leaves, all on st.
int launch_screen(Table &t, int64_t P, const uint64_t *d_vi, const uint64_t *d_vf, double k, uint64_t step_int,
                  uint64_t step_frac, const ScreenArgs &sa, ZScreen *d_z, int64_t max_hits,
                  unsigned long long *d_count, int64_t *d_hits, float *d_hsc, float *d_sc, cudaStream_t st) {
    const int nz = sa.stage_end[sa.n_stages - 1];
    MB_CUDA(cudaMemsetAsync(d_count, 0, 8, st));
    screen_prep_kernel<<<(nz + 127) / 128, 128, 0, st>>>(view(t), nz, k, step_int, step_frac, d_z);
    MB_CUDA(cudaGetLastError());
    const size_t smem = (size_t)nz * sizeof(ZScreen);
    MB_CUDA(cudaFuncSetAttribute(screen_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(SCREEN_MAX_ZEROS * sizeof(ZScreen))));
    const unsigned blocks = (unsigned)((P + SCREEN_THREADS - 1) / SCREEN_THREADS);
    screen_kernel<<<blocks, SCREEN_THREADS, smem, st>>>(d_z, nz, CandView{d_vi, d_vf, nullptr, P}, sa, max_hits,
                                                       d_count, d_hits, d_hsc, d_sc);
    MB_CUDA(cudaGetLastError());
    return MB_OK;
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" int mb_screen(mb_table *h, int64_t P, const uint64_t *v_int, const uint64_t *v_frac, double k,
                         uint64_t step_int, uint64_t step_frac, int n_stages, const int64_t *stage_end,
                         const float *threshold, int64_t max_hits, int64_t *out_hits, float *out_hit_scores,
                         int64_t *n_hits, float *out_scores) {
    const char *who = "mb_screen";
    MB_CHECK_ARG(h && v_int && v_frac && stage_end && threshold && n_hits, "%s: null argument", who);
    Table &t = table_of(h);
    MB_CHECK_ARG(max_hits >= 0 && (max_hits == 0 || (out_hits && out_hit_scores)), "%s: hit buffers", who);
    ScreenArgs sa;
    MB_TRY(screen_args(t, n_stages, stage_end, threshold, k, P, max_hits, who, sa));
    *n_hits = 0;
    if (P == 0) return MB_OK;
    MB_TRY(device_guard(t.device));
    const int nz = sa.stage_end[n_stages - 1];
    const size_t cand = (size_t)P * 8;
    const size_t sc_bytes = out_scores ? (size_t)P * n_stages * 4 : 0;
    const size_t need = 2 * (cand + 256) + (nz * sizeof(ZScreen) + 256) + 256 + ((size_t)max_hits * 8 + 256) +
                        ((size_t)max_hits * n_stages * 4 + 256) + (sc_bytes + 256);
    MB_TRY(t.io.ensure(need));
    char *q = (char *)t.io.p;
    uint64_t *d_vi = carve<uint64_t>(q, P), *d_vf = carve<uint64_t>(q, P);
    ZScreen *d_z = carve<ZScreen>(q, nz);
    unsigned long long *d_count = carve<unsigned long long>(q, 1);
    int64_t *d_hits = carve<int64_t>(q, max_hits);
    float *d_hsc = carve<float>(q, (size_t)max_hits * n_stages);
    float *d_sc = out_scores ? carve<float>(q, (size_t)P * n_stages) : nullptr;
    cudaStream_t st = t.stream;
    MB_CUDA(cudaMemcpyAsync(d_vi, v_int, cand, cudaMemcpyHostToDevice, st));
    MB_CUDA(cudaMemcpyAsync(d_vf, v_frac, cand, cudaMemcpyHostToDevice, st));
    MB_TRY(launch_screen(t, P, d_vi, d_vf, k, step_int, step_frac, sa, d_z, max_hits, d_count, d_hits, d_hsc,
                         d_sc, st));
    unsigned long long total = 0;
    MB_CUDA(cudaMemcpyAsync(&total, d_count, 8, cudaMemcpyDeviceToHost, st));
    if (out_scores) MB_CUDA(cudaMemcpyAsync(out_scores, d_sc, sc_bytes, cudaMemcpyDeviceToHost, st));
    MB_CUDA(cudaStreamSynchronize(st));
    *n_hits = (int64_t)total;
    const int64_t kept = std::min<int64_t>((int64_t)total, max_hits);
    if (kept > 0) {
        std::vector<int64_t> idx(kept);
        std::vector<float> hs((size_t)kept * n_stages);
        MB_CUDA(cudaMemcpy(idx.data(), d_hits, kept * 8, cudaMemcpyDeviceToHost));
        MB_CUDA(cudaMemcpy(hs.data(), d_hsc, (size_t)kept * n_stages * 4, cudaMemcpyDeviceToHost));
        // the atomic slots come in arbitrary order: return hits sorted by leaf index
        std::vector<int64_t> ord(kept);
        std::iota(ord.begin(), ord.end(), 0);
        std::sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) { return idx[a] < idx[b]; });
        for (int64_t i = 0; i < kept; ++i) {
            out_hits[i] = idx[ord[i]];
            for (int s = 0; s < n_stages; ++s) out_hit_scores[i * n_stages + s] = hs[ord[i] * n_stages + s];
        }
    }
    if ((int64_t)total > max_hits) {
        set_error("%s: %llu hits exceed max_hits=%lld (the kept subset is arbitrary)", who, total,
                  (long long)max_hits);
        return MB_ERR_CAPACITY;
    }
    return MB_OK;
}

extern "C" int mb_screen_dev(mb_table *h, int64_t P, const uint64_t *d_v_int, const uint64_t *d_v_frac, double k,
                             uint64_t step_int, uint64_t step_frac, int n_stages, const int64_t *stage_end,
                             const float *threshold, int64_t max_hits, int64_t *d_hits, float *d_hit_scores,
                             unsigned long long *d_n_hits, float *d_scores, void *stream) {
    const char *who = "mb_screen_dev";
    MB_CHECK_ARG(h && d_v_int && d_v_frac && d_n_hits, "%s: null argument", who);
    MB_CHECK_ARG(max_hits == 0 || (d_hits && d_hit_scores), "%s: hit buffers", who);
    Table &t = table_of(h);
    ScreenArgs sa;
    MB_TRY(screen_args(t, n_stages, stage_end, threshold, k, P, max_hits, who, sa));
    MB_TRY(device_guard(t.device));
    const cudaStream_t st = (cudaStream_t)stream;
    if (P == 0) {
        MB_CUDA(cudaMemsetAsync(d_n_hits, 0, 8, st));
        return MB_OK;
    }
    const int nz = sa.stage_end[n_stages - 1];
    MB_TRY(t.screen.ensure(nz * sizeof(ZScreen)));
    MB_TRY(launch_screen(t, P, d_v_int, d_v_frac, k, step_int, step_frac, sa, (ZScreen *)t.screen.p, max_hits,
                         d_n_hits, d_hits, d_hit_scores, d_scores, st));
    return MB_OK;
}
