// Plans for the chosen-form kernel: tier boundaries from an a-priori error bound, candidate
// tiles and zero chunks as work items (largest first), partial-sum layout, and a CUDA graph
// for repeated runs on fixed buffers.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "k2_fast.h"
#include "k2_internal.h"

using namespace mb;

struct mb_plan {
    Table *table = nullptr;
    int n_groups = 0;
    int64_t P = 0;
    double tol = 1e-10;
    std::vector<int64_t> counts;
    std::vector<double> ks, Ts;
    std::vector<int> wslot;        // per group: table weight vector, or -1 for exp(-k gamma^2)
    std::vector<FastGroup> groups;
    std::vector<FastItem> items;      // heavy items, then light items
    std::vector<FastItem> items_lpt;  // schedule 2: the same items by estimated cost, both tiers mixed
    std::vector<int64_t> n_T, n_eval, n_heavy;   // zeros below T, zeros evaluated, heavy zeros
    double skip_frac = 0.0;        // share of tol given to skipping the tail of each group
    std::vector<double> err_bound, sum_abs;
    std::vector<double> err_dd, err_dk;   // the same a-priori bounds for dK2/ddelta and dK2/dk
    std::vector<int> shape_nzw;
    std::vector<int64_t> heavy_chunk, light_chunk;
    int light_cpt = 4;
    int schedule = 0;              // 0: two concurrent tier kernels, 1: one persistent kernel,
                                   // 2: the same, cost-ordered, 3: the same, one CTA of each tier per SM
    int nzw_shift = 0;             // extra doublings of the default warps-per-candidate-set split
    double chunk_scale = 1.0;      // multiplies the automatic work-item sizes
    int64_t z_begin = 0, z_end = INT64_MAX;   // zero-range shard of every group (default: all)
    int n_heavy_items = 0;
    double zero_terms = 0;
    FastPlanDev dev;
    size_t partial_doubles = 0;
    // host-pointer runs: device candidate/result buffers, pinned staging and a captured graph
    uint64_t *d_vi = nullptr, *d_vf = nullptr;
    double *d_delta = nullptr, *d_out = nullptr;
    void *h_pinned = nullptr;
    cudaGraphExec_t graph = nullptr;
    DevBuf newton_buf;             // Newton polish: starting point, its gradients, stop flags
    DevBuf flush_buf;              // mb_plan_time: written between timed runs to empty the L2
    // per-kernel timing hook (mb_plan_kernel_timing): a ring of event sets, one per device run
    std::vector<TierEvents> tev;
    std::vector<signed char> tev_tiers;   // tiers each slot's run launched (bit 0 heavy, 1 light)
    long long tev_runs = 0;
    void release_events() {
        for (TierEvents &e : tev) {
            cudaEventDestroy(e.light0);
            cudaEventDestroy(e.light1);
            cudaEventDestroy(e.heavy0);
            cudaEventDestroy(e.heavy1);
        }
        tev.clear();
        tev_tiers.clear();
        tev_runs = 0;
    }
    ~mb_plan() {
        newton_buf.release();
        flush_buf.release();
        release_events();
    }
};

namespace {

void free_dev(mb_plan *p) {
    if (p->dev.items_one != p->dev.items) cudaFree(p->dev.items_one);
    cudaFree(p->dev.items);
    cudaFree(p->dev.groups);
    cudaFree(p->dev.counter);
    cudaFree(p->dev.partial);
    p->dev = FastPlanDev();
}

void free_io(mb_plan *p) {
    if (p->graph) cudaGraphExecDestroy(p->graph);
    p->graph = nullptr;
    cudaFree(p->d_vi);
    cudaFree(p->d_vf);
    cudaFree(p->d_delta);
    cudaFree(p->d_out);
    if (p->h_pinned) cudaFreeHost(p->h_pinned);
    p->d_vi = p->d_vf = nullptr;
    p->d_delta = p->d_out = nullptr;
    p->h_pinned = nullptr;
}

// Default number of warps splitting one candidate set's zeros, so that a candidate tile
// ((8/nzw) * 32 * cpt candidates) is not much larger than the group.
int default_nzw(int64_t P, int cpt) {
    int nzw = 1;
    while (nzw < 8 && (int64_t)(8 / nzw) * 32 * cpt > 2 * P) nzw *= 2;
    return nzw;
}

// Tier boundary and tail skip, with a_j = 2|c_j| w_j >= |term_j| (w_j = exp(-k gamma_j^2) or the
// group's weight vector):
//   n_eval: the smallest n with sum_{n <= j < n_use} a_j <= skip_frac * tol -- those zeros are
//           not evaluated (skip_frac = 0: every zero below T is evaluated);
//   n_h:    the smallest n_h that keeps the whole bound (skipped sum + EPS_LIGHT * light sum +
//           EPS_HEAVY * heavy sum + FP64 roundings) within 0.99 tol.
// Returns the a-priori bound of |K2 error| (skipped sum + tier errors + FP64 roundings).
void plan_tiers(const Table &t, int64_t n_use, double k, const double *wts, double tol, double skip_frac,
                int64_t &n_eval, int64_t &n_h, double &bound, double &sabs, double &bound_dd, double &bound_dk) {
    std::vector<double> a(n_use);
    double total = 0;
    for (int64_t j = 0; j < n_use; ++j) {
        double g = t.h_gamma[j];
        a[j] = 2.0 * t.h_alpha[j] * (wts ? std::fabs(wts[j]) : std::exp(-k * g * g));
        total += a[j];
    }
    double skipped = 0;
    n_eval = n_use;
    if (skip_frac > 0)
        for (int64_t j = n_use - 1; j >= 0; --j) {
            if (skipped + a[j] > skip_frac * tol) break;
            skipped += a[j];
            n_eval = j;
        }
    // The light tier takes zeros from the top while the whole bound stays within 0.99 tol
    // (the heavy tier's and the roundings' shares are tiny, so nearly all of the rest of tol).
    // FP64 accumulation and reduction of the heavy sum and of the light partials: at most
    // ~(terms per thread + chunks) roundings of 2^-53 relative; 1e-13 relative is a safe cover.
    const double evaluated = total - skipped;
    const double fixed = skipped + 1e-13 * evaluated;
    double tail = 0;
    n_h = n_eval;
    for (int64_t j = n_eval - 1; j >= 0; --j) {
        const double t2 = tail + a[j];
        if (fixed + EPS_LIGHT * t2 + EPS_HEAVY * (evaluated - t2) > 0.99 * tol) break;
        tail = t2;
        n_h = j;
    }
    double heavy = evaluated - tail;
    bound = fixed + EPS_LIGHT * tail + EPS_HEAVY * heavy;
    sabs = total;
    // the derivative terms are the value terms with amplitudes a gamma and a gamma^2 (computed
    // the same way in each tier), so the same per-unit errors apply to those amplitude sums
    double s1[3] = {0, 0, 0}, s2[3] = {0, 0, 0};       // [heavy, light, skipped]
    for (int64_t j = 0; j < n_use; ++j) {
        const int tier = j < n_h ? 0 : (j < n_eval ? 1 : 2);
        const double g = t.h_gamma[j];
        s1[tier] += a[j] * g;
        s2[tier] += a[j] * g * g;
    }
    bound_dd = s1[2] + EPS_LIGHT * s1[1] + EPS_HEAVY * s1[0] + 1e-13 * (s1[0] + s1[1]);
    bound_dk = s2[2] + EPS_LIGHT * s2[1] + EPS_HEAVY * s2[0] + 1e-13 * (s2[0] + s2[1]);
}

void replan_tiers(mb_plan *p) {
    const Table &t = *p->table;
    for (int g = 0; g < p->n_groups; ++g) {
        const double *wh = p->wslot[g] >= 0 ? t.h_weights[p->wslot[g]].data() : nullptr;
        plan_tiers(t, p->n_T[g], p->ks[g], wh, p->tol, p->skip_frac, p->n_eval[g], p->n_heavy[g],
                   p->err_bound[g], p->sum_abs[g], p->err_dd[g], p->err_dk[g]);
    }
}

// Work items.  Heavy items (FP64 tier) use HEAVY_CPT candidates per thread and are pulled by
// the persistent heavy kernel (two CTAs per SM); light items use the plan's light_cpt and run
// one CTA each.  Chunk sizes aim at ~4 heavy items and ~18 light items per SM.
int build_items(mb_plan *p, int sms) {
    p->groups.clear();
    p->items.clear();
    p->zero_terms = 0;
    // the zeros this plan evaluates: [zb, ze) within each group's [0, n_T) (a zero-range shard)
    auto hb = [&](int g) { return std::max<int64_t>(0, p->z_begin); };
    auto he = [&](int g) { return std::min(p->n_heavy[g], p->z_end); };
    auto lb = [&](int g) { return std::max(p->n_heavy[g], p->z_begin); };
    auto le = [&](int g) { return std::min(p->n_eval[g], p->z_end); };
    double Wh = 0, Wl = 0;
    for (int g = 0; g < p->n_groups; ++g) {
        Wh += (double)p->counts[g] * std::max<int64_t>(0, he(g) - hb(g));
        Wl += (double)p->counts[g] * std::max<int64_t>(0, le(g) - lb(g));
    }
    // ~4 heavy items per SM (two per heavy CTA) and ~18 light items per SM (several waves)
    const double target_h = std::max(p->chunk_scale * Wh / (4.0 * sms), 1.0);
    const double target_l = std::max(p->chunk_scale * Wl / (18.0 * sms), 1.0);
    std::vector<FastItem> heavy, light;
    int64_t c0 = 0, pbase = 0;
    for (int g = 0; g < p->n_groups; ++g) {
        FastGroup gr{};
        gr.c0 = c0;
        gr.nc = p->counts[g];
        gr.k = p->ks[g];
        gr.w = p->wslot[g] >= 0 ? p->table->d_weights[p->wslot[g]] : nullptr;
        gr.pbase = pbase;
        const int nzw = p->shape_nzw[g];
        const int64_t CTh = (int64_t)(8 / nzw) * 32 * HEAVY_CPT;
        const int64_t CTl = (int64_t)(8 / nzw) * 32 * p->light_cpt;
        int64_t hz = p->heavy_chunk[g], lz = p->light_chunk[g];
        // chunk = target terms / tile candidates, rounded to whole tiles (at least 1 heavy tile of
        // 128 zeros and 8 light tiles of 256: finer heavy items balance the persistent kernel,
        // coarser light items cost less per term -- both measured)
        if (hz <= 0)
            hz = std::max<int64_t>(128, ((int64_t)(target_h / std::min<int64_t>(CTh, std::max<int64_t>(gr.nc, 1))) + 64) / 128 * 128);
        // the last light chunks of a group are a quarter of the size, about one round of CTA slots
        // in all (this group's share of it), so the light items' last wave -- they run largest
        // first -- ends in small items instead of leaving SMs idle behind full-size ones
        int64_t small_lz = 0, small_from = le(g);
        if (lz <= 0) {
            lz = std::max<int64_t>(2048, ((int64_t)(target_l / std::min<int64_t>(CTl, std::max<int64_t>(gr.nc, 1))) + 128) / 256 * 256);
            const int per_sm = p->light_cpt == 2 ? 4 : (p->light_cpt == 3 ? 3 : 2);
            const double wg = (double)gr.nc * std::max<int64_t>(0, le(g) - lb(g));
            const int64_t n_tiles = std::max<int64_t>(1, (gr.nc + CTl - 1) / CTl);
            const int64_t items = (int64_t)std::ceil((double)sms * per_sm * (Wl > 0 ? wg / Wl : 0.0));
            small_lz = std::max<int64_t>(256, lz / 4 / 256 * 256);
            const int64_t span = ((items + n_tiles - 1) / n_tiles) * small_lz;
            if (span > 0 && le(g) - lb(g) > 2 * span) small_from = le(g) - span;
        }
        int ch = 0;
        auto emit = [&](int64_t z0, int64_t z1, int tier, int64_t CT, int cpt, std::vector<FastItem> &dst) {
            for (int64_t ct = 0; ct * CT < gr.nc; ++ct) {
                FastItem it{};
                it.c0 = c0 + ct * CT;
                it.nc = (int)std::min<int64_t>(CT, gr.nc - ct * CT);
                it.group = g;
                it.z0 = z0;
                it.z1 = z1;
                it.pbase = pbase + (int64_t)ch * gr.nc * 3;
                it.tier = tier;
                it.cpt = cpt;
                it.nzw = nzw;
                dst.push_back(it);
            }
            ++ch;
        };
        for (int64_t z = hb(g); z < he(g); z += hz)
            emit(z, std::min(z + hz, he(g)), 0, CTh, HEAVY_CPT, heavy);
        for (int64_t z = lb(g); z < small_from; z += lz)
            emit(z, std::min(z + lz, small_from), 1, CTl, p->light_cpt, light);
        for (int64_t z = small_from; z < le(g); z += small_lz)
            emit(z, std::min(z + small_lz, le(g)), 1, CTl, p->light_cpt, light);
        gr.n_chunks = ch;
        p->zero_terms += (double)gr.nc * (std::max<int64_t>(0, he(g) - hb(g)) + std::max<int64_t>(0, le(g) - lb(g)));
        pbase += (int64_t)gr.n_chunks * gr.nc * 3;
        c0 += gr.nc;
        p->groups.push_back(gr);
    }
    auto by_cost = [](const FastItem &a, const FastItem &b) {
        return (double)a.nc * (a.z1 - a.z0) > (double)b.nc * (b.z1 - b.z0);
    };
    std::stable_sort(heavy.begin(), heavy.end(), by_cost);
    std::stable_sort(light.begin(), light.end(), by_cost);
    p->n_heavy_items = (int)heavy.size();
    if (p->schedule == 2) {
        // one kernel, every item of both tiers in one list, largest estimated cost first (a heavy
        // term costs ~2.5 light terms, measured alone): the longest-processing-time order, so the
        // last items to start, of either tier, are the smallest
        auto cost = [](const FastItem &a) { return (a.tier == 0 ? 2.5 : 1.0) * a.nc * (double)(a.z1 - a.z0); };
        p->items_lpt = heavy;
        p->items_lpt.insert(p->items_lpt.end(), light.begin(), light.end());
        std::stable_sort(p->items_lpt.begin(), p->items_lpt.end(),
                         [&](const FastItem &a, const FastItem &b) { return cost(a) > cost(b); });
    } else {
        p->items_lpt.clear();
    }
    // heavy items then light items: the two-kernel schedule and every one-tier run use this order
    p->items = heavy;
    p->items.insert(p->items.end(), light.begin(), light.end());
    p->partial_doubles = (size_t)std::max<int64_t>(pbase, 3);
    return MB_OK;
}

int upload(mb_plan *p) {
    free_dev(p);
    free_io(p);
    MB_TRY(device_guard(p->table->device));
    MB_TRY(heavy_smem_attributes());
    int sms = 148;
    MB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->table->device));
    MB_TRY(build_items(p, sms));
    MB_CUDA(cudaMalloc(&p->dev.items, std::max<size_t>(1, p->items.size()) * sizeof(FastItem)));
    MB_CUDA(cudaMalloc(&p->dev.groups, std::max<size_t>(1, p->groups.size()) * sizeof(FastGroup)));
    MB_CUDA(cudaMalloc(&p->dev.counter, TIERS_COUNTERS * sizeof(int)));
    MB_CUDA(cudaMalloc(&p->dev.partial, p->partial_doubles * sizeof(double)));
    p->dev.partial_bytes = p->partial_doubles * sizeof(double);
    if (!p->items.empty())
        MB_CUDA(cudaMemcpy(p->dev.items, p->items.data(), p->items.size() * sizeof(FastItem), cudaMemcpyHostToDevice));
    p->dev.items_one = p->dev.items;
    if (!p->items_lpt.empty()) {
        MB_CUDA(cudaMalloc(&p->dev.items_one, p->items_lpt.size() * sizeof(FastItem)));
        MB_CUDA(cudaMemcpy(p->dev.items_one, p->items_lpt.data(), p->items_lpt.size() * sizeof(FastItem),
                           cudaMemcpyHostToDevice));
    }
    MB_CUDA(cudaMemcpy(p->dev.groups, p->groups.data(), p->groups.size() * sizeof(FastGroup), cudaMemcpyHostToDevice));
    p->dev.n_heavy = p->n_heavy_items;
    p->dev.n_light = (int)p->items.size() - p->n_heavy_items;
    p->dev.n_groups = (int)p->groups.size();
    p->dev.light_cpt = p->light_cpt;
    p->dev.one_kernel = p->schedule >= 1;
    p->dev.paired = p->schedule == 3;
    p->dev.fused_phase = p->table->h_gamma.empty() || p->table->h_gamma.back() < FUSED_PHASE_GAMMA;
    unsigned hg = 148;
    MB_TRY(heavy_grid_size(p->table->device, &hg));
    p->dev.heavy_grid = std::min<unsigned>(hg, (unsigned)std::max(1, p->n_heavy_items));
    p->dev.tiers_grid = std::min<unsigned>(hg, (unsigned)std::max<size_t>(1, p->items.size()));
    return MB_OK;
}

int plan_run_dev(mb_plan *p, const uint64_t *vi, const uint64_t *vf, const double *delta, double *val,
                 double *dd, double *dk, cudaStream_t s) {
    return launch_fast(*p->table, p->dev, CandView{vi, vf, delta, p->P}, val, dd, dk, s);
}

// A device-pointer run that records the timing hook's events when it is on (never inside the
// plan's own graph capture: ensure_io calls plan_run_dev directly).
int plan_run_timed(mb_plan *p, int tiers, const uint64_t *vi, const uint64_t *vf, const double *delta,
                   double *val, double *dd, double *dk, cudaStream_t s) {
    const TierEvents *ev = nullptr;
    if (!p->tev.empty()) {
        const size_t slot = (size_t)(p->tev_runs % (long long)p->tev.size());
        ev = &p->tev[slot];
        int ran = ((tiers & 1) && p->dev.n_heavy > 0 ? 1 : 0) | ((tiers & 2) && p->dev.n_light > 0 ? 2 : 0);
        if (ran == 3 && p->dev.one_kernel) ran = 2;      // one kernel: its time is the light pair
        p->tev_tiers[slot] = (signed char)ran;
        ++p->tev_runs;
    }
    return launch_fast(*p->table, p->dev, CandView{vi, vf, delta, p->P}, val, dd, dk, s, tiers, ev);
}

int ensure_io(mb_plan *p) {
    if (p->d_out) return MB_OK;
    size_t P = (size_t)std::max<int64_t>(p->P, 1);
    MB_CUDA(cudaMalloc(&p->d_vi, P * 8));
    MB_CUDA(cudaMalloc(&p->d_vf, P * 8));
    MB_CUDA(cudaMalloc(&p->d_delta, P * 8));
    MB_CUDA(cudaMalloc(&p->d_out, 3 * P * 8));
    MB_CUDA(cudaHostAlloc(&p->h_pinned, 6 * P * 8, cudaHostAllocDefault));
    // capture: H2D of the candidates, the kernels, D2H of the results
    cudaStream_t s = p->table->stream;
    char *h = (char *)p->h_pinned;
    MB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync(p->d_vi, h, P * 8, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(p->d_vf, h + P * 8, P * 8, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(p->d_delta, h + 2 * P * 8, P * 8, cudaMemcpyHostToDevice, s);
    int st = plan_run_dev(p, p->d_vi, p->d_vf, p->d_delta, p->d_out, p->d_out + P, p->d_out + 2 * P, s);
    cudaMemcpyAsync(h + 3 * P * 8, p->d_out, 3 * P * 8, cudaMemcpyDeviceToHost, s);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (st != MB_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) {
        set_error("plan graph capture: %s", cudaGetErrorString(e));
        return MB_ERR_CUDA;
    }
    e = cudaGraphInstantiate(&p->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        set_error("plan graph instantiate: %s", cudaGetErrorString(e));
        return MB_ERR_CUDA;
    }
    return MB_OK;
}

}  // namespace

extern "C" int mb_plan_create_weighted(mb_table *h, int n_groups, const int64_t *counts, const double *ks,
                                       const double *Ts, const int *weight_slots, double tol, mb_plan **out) {
    MB_CHECK_ARG(out != nullptr, "mb_plan_create: out is null");
    *out = nullptr;
    MB_CHECK_ARG(h && counts && ks && Ts, "mb_plan_create: null argument");
    MB_CHECK_ARG(n_groups >= 1 && n_groups <= 4096, "mb_plan_create: n_groups=%d", n_groups);
    MB_CHECK_ARG(std::isfinite(tol) && tol > 0, "mb_plan_create: tol=%g must be > 0", tol);
    Table &t = table_of(h);
    int64_t P = 0;
    for (int g = 0; g < n_groups; ++g) {
        MB_CHECK_ARG(counts[g] >= 0 && counts[g] <= ((int64_t)1 << 26), "mb_plan_create: count[%d]", g);
        MB_CHECK_ARG(std::isfinite(ks[g]) && ks[g] >= 0, "mb_plan_create: k[%d]=%g", g, ks[g]);
        MB_CHECK_ARG(!std::isnan(Ts[g]), "mb_plan_create: T[%d] is NaN", g);
        if (weight_slots)
            MB_CHECK_ARG(weight_slots[g] >= -1 && weight_slots[g] < (int)t.d_weights.size(),
                         "mb_plan_create: weight slot %d of group %d not registered", weight_slots[g], g);
        P += counts[g];
    }
    MB_CHECK_ARG(P <= ((int64_t)1 << 26), "mb_plan_create: total P=%lld too large", (long long)P);
    MB_TRY(device_guard(t.device));
    mb_plan *p = new mb_plan();
    p->table = &t;
    p->n_groups = n_groups;
    p->P = P;
    p->tol = tol;
    p->counts.assign(counts, counts + n_groups);
    p->ks.assign(ks, ks + n_groups);
    p->Ts.assign(Ts, Ts + n_groups);
    p->n_T.resize(n_groups);
    p->n_eval.resize(n_groups);
    p->n_heavy.resize(n_groups);
    p->err_bound.resize(n_groups);
    p->sum_abs.resize(n_groups);
    p->err_dd.resize(n_groups);
    p->err_dk.resize(n_groups);
    p->shape_nzw.resize(n_groups);
    p->heavy_chunk.assign(n_groups, 0);
    p->light_chunk.assign(n_groups, 0);
    p->wslot.assign(n_groups, -1);
    if (weight_slots) p->wslot.assign(weight_slots, weight_slots + n_groups);
    for (int g = 0; g < n_groups; ++g) {
        p->n_T[g] = t.count_below(Ts[g]);
        p->shape_nzw[g] = default_nzw(counts[g], p->light_cpt);
    }
    replan_tiers(p);
    int st = upload(p);
    if (st != MB_OK) {
        free_dev(p);
        delete p;
        return st;
    }
    ++t.n_plans;
    *out = p;
    return MB_OK;
}

extern "C" int mb_plan_create(mb_table *h, int n_groups, const int64_t *counts, const double *ks,
                              const double *Ts, double tol, mb_plan **out) {
    return mb_plan_create_weighted(h, n_groups, counts, ks, Ts, nullptr, tol, out);
}

extern "C" int mb_plan_destroy(mb_plan *p) {
    if (!p) return MB_OK;
    device_guard(p->table->device);
    free_io(p);
    free_dev(p);
    --p->table->n_plans;
    delete p;
    return MB_OK;
}

extern "C" int mb_plan_set_shape(mb_plan *p, int g, int cpt, int nzw, int64_t heavy_chunk,
                                 int64_t light_chunk) {
    MB_CHECK_ARG(p && g >= 0 && g < p->n_groups, "mb_plan_set_shape: bad plan/group");
    MB_CHECK_ARG(cpt == 2 || cpt == 3 || cpt == 4, "mb_plan_set_shape: light cpt=%d (2, 3 or 4)", cpt);
    MB_CHECK_ARG(nzw == 1 || nzw == 2 || nzw == 4 || nzw == 8, "mb_plan_set_shape: nzw=%d", nzw);
    MB_CHECK_ARG(heavy_chunk == 0 || (heavy_chunk > 0 && heavy_chunk % 128 == 0), "mb_plan_set_shape: heavy_chunk");
    MB_CHECK_ARG(light_chunk == 0 || (light_chunk > 0 && light_chunk % 256 == 0), "mb_plan_set_shape: light_chunk");
    p->light_cpt = cpt;    // plan-wide: the light kernel is instantiated per candidates-per-thread
    p->shape_nzw[g] = nzw;
    p->heavy_chunk[g] = heavy_chunk;
    p->light_chunk[g] = light_chunk;
    MB_TRY(device_guard(p->table->device));
    return upload(p);
}

// Plan-wide tile configuration (the autotuner's search space): light_cpt candidates per thread
// in the light kernel (2, 3, 4), nzw_shift extra doublings of every group's warp split (0..3,
// capped at 8 warps), chunk_scale times the automatic work-item size (0.125 .. 8).  Per-group
// overrides set with mb_plan_set_shape are replaced.
extern "C" int mb_plan_configure(mb_plan *p, int light_cpt, int nzw_shift, double chunk_scale) {
    MB_CHECK_ARG(p, "mb_plan_configure: null plan");
    MB_CHECK_ARG(light_cpt == 2 || light_cpt == 3 || light_cpt == 4, "mb_plan_configure: light_cpt=%d", light_cpt);
    MB_CHECK_ARG(nzw_shift >= 0 && nzw_shift <= 3, "mb_plan_configure: nzw_shift=%d", nzw_shift);
    MB_CHECK_ARG(chunk_scale >= 0.125 && chunk_scale <= 8.0, "mb_plan_configure: chunk_scale=%g", chunk_scale);
    p->light_cpt = light_cpt;
    p->nzw_shift = nzw_shift;
    p->chunk_scale = chunk_scale;
    for (int g = 0; g < p->n_groups; ++g) {
        p->shape_nzw[g] = std::min(8, default_nzw(p->counts[g], light_cpt) << nzw_shift);
        p->heavy_chunk[g] = 0;
        p->light_chunk[g] = 0;
    }
    MB_TRY(device_guard(p->table->device));
    return upload(p);
}

extern "C" int mb_plan_set_schedule(mb_plan *p, int schedule) {
    MB_CHECK_ARG(p, "mb_plan_set_schedule: null plan");
    MB_CHECK_ARG(schedule >= 0 && schedule <= 3, "mb_plan_set_schedule: schedule=%d (0 .. 3)", schedule);
    MB_TRY(device_guard(p->table->device));
    const bool reorder = (schedule == 2) != (p->schedule == 2);
    p->schedule = schedule;
    if (reorder) return upload(p);     // the item order changes
    p->dev.one_kernel = schedule >= 1;
    p->dev.paired = schedule == 3;
    free_io(p);                    // the captured graph holds the old launch sequence
    return MB_OK;
}

extern "C" int mb_plan_schedule(const mb_plan *p, int *schedule) {
    MB_CHECK_ARG(p && schedule, "mb_plan_schedule: null argument");
    *schedule = p->schedule;
    return MB_OK;
}

// Give the share skip_frac (0 .. 1/4) of tol to not evaluating each group's negligible tail: the
// zeros beyond the point where the remaining sum of 2|c| w is <= skip_frac tol are skipped, and
// the light tier fits in what remains of tol.  The bound of mb_plan_group_info includes the
// skipped sum.  (The derivative outputs then omit sum 2|c| w gamma and 2|c| w gamma^2 over the
// same zeros.)  0 restores the evaluation of every zero below T.
extern "C" int mb_plan_set_skip(mb_plan *p, double skip_frac) {
    MB_CHECK_ARG(p, "mb_plan_set_skip: null plan");
    MB_CHECK_ARG(skip_frac >= 0.0 && skip_frac <= 0.25, "mb_plan_set_skip: skip_frac=%g (0 .. 0.25)", skip_frac);
    p->skip_frac = skip_frac;
    replan_tiers(p);
    MB_TRY(device_guard(p->table->device));
    return upload(p);
}

extern "C" int mb_plan_group_bounds(const mb_plan *p, int g, double *val, double *dd, double *dk) {
    MB_CHECK_ARG(p && g >= 0 && g < p->n_groups, "mb_plan_group_bounds: bad plan/group");
    if (val) *val = p->err_bound[g];
    if (dd) *dd = p->err_dd[g];
    if (dk) *dk = p->err_dk[g];
    return MB_OK;
}

extern "C" int mb_plan_group_zeros(const mb_plan *p, int g, int64_t *n_eval) {
    MB_CHECK_ARG(p && n_eval && g >= 0 && g < p->n_groups, "mb_plan_group_zeros: bad plan/group");
    *n_eval = p->n_eval[g];
    return MB_OK;
}

// Restrict every group to the zeros [j0, j1) (intersected with its [0, n_T)): a zero-range shard.
// Tier boundaries and error bounds stay those of the whole sum; the shards' results add up to it.
extern "C" int mb_plan_set_zero_range(mb_plan *p, int64_t j0, int64_t j1) {
    MB_CHECK_ARG(p, "mb_plan_set_zero_range: null plan");
    MB_CHECK_ARG(0 <= j0 && j0 <= j1, "mb_plan_set_zero_range: [%lld, %lld)", (long long)j0, (long long)j1);
    p->z_begin = j0;
    p->z_end = j1;
    MB_TRY(device_guard(p->table->device));
    return upload(p);
}

// Median device time (ms) of `reps` runs of the plan on synthetic candidates (the values do not
// change the work), after one warm-up run, each run after a 192 MB write that empties the L2.
// Used by the autotuner.
extern "C" int mb_plan_time(mb_plan *p, int reps, double *ms) {
    MB_CHECK_ARG(p && ms && reps >= 1 && reps <= 1000, "mb_plan_time: bad argument");
    MB_TRY(device_guard(p->table->device));
    if (p->P == 0) {
        *ms = 0.0;
        return MB_OK;
    }
    MB_TRY(ensure_io(p));
    const size_t P = (size_t)p->P;
    std::vector<uint64_t> v(2 * P);
    uint64_t x = 0x9E3779B97F4A7C15ull;
    for (size_t i = 0; i < 2 * P; ++i) {
        x ^= x << 13; x ^= x >> 7; x ^= x << 17;
        v[i] = (i < P) ? 3400000000000000000ull + (x % 200000000000000000ull) : x;
    }
    cudaStream_t s = p->table->stream;
    MB_CUDA(cudaMemcpyAsync(p->d_vi, v.data(), P * 8, cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaMemcpyAsync(p->d_vf, v.data() + P, P * 8, cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaMemsetAsync(p->d_delta, 0, P * 8, s));
    // each timed run starts from an empty L2 (the 126 MB L2 would otherwise keep the table)
    const size_t flush_bytes = (size_t)192 << 20;
    MB_TRY(p->flush_buf.ensure(flush_bytes));
    cudaEvent_t e0, e1;
    MB_CUDA(cudaEventCreate(&e0));
    MB_CUDA(cudaEventCreate(&e1));
    std::vector<float> t;
    int st = plan_run_dev(p, p->d_vi, p->d_vf, p->d_delta, p->d_out, p->d_out + P, p->d_out + 2 * P, s);
    for (int r = 0; r < reps && st == MB_OK; ++r) {
        if (cudaMemsetAsync(p->flush_buf.p, r & 0xff, flush_bytes, s) != cudaSuccess) {
            st = MB_ERR_CUDA;
            set_error("mb_plan_time: L2 flush failed");
            break;
        }
        cudaEventRecord(e0, s);
        st = plan_run_dev(p, p->d_vi, p->d_vf, p->d_delta, p->d_out, p->d_out + P, p->d_out + 2 * P, s);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float m = 0;
        cudaEventElapsedTime(&m, e0, e1);
        t.push_back(m);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    MB_TRY(st);
    MB_CUDA(cudaGetLastError());
    std::sort(t.begin(), t.end());
    *ms = t[t.size() / 2];
    return MB_OK;
}

// The autotuner's search: every (light_cpt, nzw_shift, chunk_scale) in {2, 3, 4} x {0, 1} x
// {0.5, 1, 2} (in that nesting order) timed by mb_plan_time(reps); the fastest is applied.
extern "C" int mb_plan_autotune(mb_plan *p, int reps, int *light_cpt, int *nzw_shift, double *chunk_scale,
                                double *best_ms, double *timings) {
    MB_CHECK_ARG(p && reps >= 1 && reps <= 1000, "mb_plan_autotune: bad argument");
    static const int cpts[3] = {2, 3, 4};
    static const int shifts[2] = {0, 1};
    static const double scales[3] = {0.5, 1.0, 2.0};
    int bc = 4, bs = 0;
    double bsc = 1.0, bms = INFINITY;
    int i = 0;
    for (int c : cpts)
        for (int sh : shifts)
            for (double sc : scales) {
                MB_TRY(mb_plan_configure(p, c, sh, sc));
                double ms = 0;
                MB_TRY(mb_plan_time(p, reps, &ms));
                if (timings) timings[i] = ms;
                ++i;
                if (ms < bms) {
                    bms = ms;
                    bc = c;
                    bs = sh;
                    bsc = sc;
                }
            }
    MB_TRY(mb_plan_configure(p, bc, bs, bsc));
    if (light_cpt) *light_cpt = bc;
    if (nzw_shift) *nzw_shift = bs;
    if (chunk_scale) *chunk_scale = bsc;
    if (best_ms) *best_ms = bms;
    return MB_OK;
}

extern "C" int mb_plan_info(const mb_plan *p, int64_t *P, double *zero_terms, int *n_items) {
    MB_CHECK_ARG(p, "mb_plan_info: null plan");
    if (P) *P = p->P;
    if (zero_terms) *zero_terms = p->zero_terms;
    if (n_items) *n_items = (int)p->items.size();
    return MB_OK;
}

extern "C" int mb_plan_light_form(const mb_plan *p, int *fused) {
    MB_CHECK_ARG(p && fused, "mb_plan_light_form: null argument");
    *fused = p->dev.fused_phase ? 1 : 0;
    return MB_OK;
}

extern "C" int mb_plan_group_info(const mb_plan *p, int g, int64_t *n_T, int64_t *n_heavy,
                                  double *err_bound, double *sum_abs) {
    MB_CHECK_ARG(p && g >= 0 && g < p->n_groups, "mb_plan_group_info: bad plan/group");
    if (n_T) *n_T = p->n_T[g];
    if (n_heavy) *n_heavy = p->n_heavy[g];
    if (err_bound) *err_bound = p->err_bound[g];
    if (sum_abs) *sum_abs = p->sum_abs[g];
    return MB_OK;
}

extern "C" int mb_plan_run_dev(mb_plan *p, const uint64_t *d_vi, const uint64_t *d_vf,
                               const double *d_delta, double *d_val, double *d_dd, double *d_dk,
                               void *stream) {
    MB_CHECK_ARG(p && d_vi && d_vf && d_val && d_dd && d_dk, "mb_plan_run_dev: null argument");
    MB_TRY(device_guard(p->table->device));
    return plan_run_timed(p, 3, d_vi, d_vf, d_delta, d_val, d_dd, d_dk, (cudaStream_t)stream);
}

extern "C" int mb_plan_run_tiers_dev(mb_plan *p, int tiers, const uint64_t *d_vi, const uint64_t *d_vf,
                                     const double *d_delta, double *d_val, double *d_dd, double *d_dk,
                                     void *stream) {
    MB_CHECK_ARG(p && d_vi && d_vf && d_val && d_dd && d_dk, "mb_plan_run_tiers_dev: null argument");
    MB_CHECK_ARG(tiers >= 1 && tiers <= 3, "mb_plan_run_tiers_dev: tiers=%d (1 heavy, 2 light, 3 both)", tiers);
    MB_TRY(device_guard(p->table->device));
    return plan_run_timed(p, tiers, d_vi, d_vf, d_delta, d_val, d_dd, d_dk, (cudaStream_t)stream);
}

extern "C" int mb_plan_kernel_timing(mb_plan *p, int n_slots) {
    MB_CHECK_ARG(p && n_slots >= 0 && n_slots <= 100000, "mb_plan_kernel_timing: bad argument (n_slots=%d)",
                 n_slots);
    MB_TRY(device_guard(p->table->device));
    // runs still in flight may record the old events: wait for them before destroying any
    if (!p->tev.empty()) MB_CUDA(cudaDeviceSynchronize());
    p->release_events();
    p->tev.resize((size_t)n_slots);
    p->tev_tiers.assign((size_t)n_slots, 0);
    for (TierEvents &e : p->tev) {
        cudaError_t r = cudaEventCreate(&e.light0);
        if (r == cudaSuccess) r = cudaEventCreate(&e.light1);
        if (r == cudaSuccess) r = cudaEventCreate(&e.heavy0);
        if (r == cudaSuccess) r = cudaEventCreate(&e.heavy1);
        if (r != cudaSuccess) {
            p->release_events();
            set_error("mb_plan_kernel_timing: %s", cudaGetErrorString(r));
            return MB_ERR_CUDA;
        }
    }
    return MB_OK;
}

extern "C" int mb_plan_kernel_times(mb_plan *p, int n, double *light_ms, double *heavy_ms, int *n_out) {
    MB_CHECK_ARG(p && n >= 0 && n_out, "mb_plan_kernel_times: bad argument");
    MB_CHECK_ARG(n == 0 || (light_ms && heavy_ms), "mb_plan_kernel_times: null output");
    MB_TRY(device_guard(p->table->device));
    const long long slots = (long long)p->tev.size();
    const long long have = std::min<long long>(std::min<long long>(p->tev_runs, slots), n);
    *n_out = (int)have;
    for (long long i = 0; i < have; ++i) {
        const long long run = p->tev_runs - have + i;
        const size_t slot = (size_t)(run % slots);
        const TierEvents &e = p->tev[slot];
        float ms = -1.f;
        light_ms[i] = heavy_ms[i] = -1.0;
        if (p->tev_tiers[slot] & 2) {
            MB_CUDA(cudaEventSynchronize(e.light1));
            MB_CUDA(cudaEventElapsedTime(&ms, e.light0, e.light1));
            light_ms[i] = ms;
        }
        if (p->tev_tiers[slot] & 1) {
            MB_CUDA(cudaEventSynchronize(e.heavy1));
            MB_CUDA(cudaEventElapsedTime(&ms, e.heavy0, e.heavy1));
            heavy_ms[i] = ms;
        }
    }
    return MB_OK;
}

extern "C" int mb_plan_tier_terms(const mb_plan *p, double *heavy_terms, double *light_terms) {
    MB_CHECK_ARG(p, "mb_plan_tier_terms: null plan");
    double h = 0, l = 0;
    for (int g = 0; g < p->n_groups; ++g) {
        h += (double)p->counts[g] * p->n_heavy[g];
        l += (double)p->counts[g] * (p->n_eval[g] - p->n_heavy[g]);
    }
    if (heavy_terms) *heavy_terms = h;
    if (light_terms) *light_terms = l;
    return MB_OK;
}

extern "C" int mb_calibrate_issue(int device, double *thread_inst_per_s) {
    MB_CHECK_ARG(thread_inst_per_s, "mb_calibrate_issue: null output");
    MB_TRY(device_guard(device));
    return calibrate_issue(device, thread_inst_per_s);
}

extern "C" int mb_calibrate_pipes(int device, double *ffma_per_s, double *mufu_per_s, double *dfma_per_s) {
    MB_CHECK_ARG(ffma_per_s || mufu_per_s || dfma_per_s, "mb_calibrate_pipes: no output");
    MB_TRY(device_guard(device));
    return calibrate_pipes(device, ffma_per_s, mufu_per_s, dfma_per_s);
}

extern "C" int mb_plan_run(mb_plan *p, const uint64_t *vi, const uint64_t *vf, const double *delta,
                           double *val, double *dd, double *dk) {
    MB_CHECK_ARG(p && vi && vf && val, "mb_plan_run: null argument");
    MB_TRY(device_guard(p->table->device));
    if (p->P == 0) return MB_OK;
    if (delta)
        for (int64_t i = 0; i < p->P; ++i)
            MB_CHECK_ARG(std::isfinite(delta[i]) && std::fabs(delta[i]) < 4.0e18, "mb_plan_run: delta[%lld]", (long long)i);
    MB_TRY(ensure_io(p));
    size_t P = (size_t)p->P;
    char *h = (char *)p->h_pinned;
    std::memcpy(h, vi, P * 8);
    std::memcpy(h + P * 8, vf, P * 8);
    if (delta) std::memcpy(h + 2 * P * 8, delta, P * 8);
    else std::memset(h + 2 * P * 8, 0, P * 8);
    MB_CUDA(cudaGraphLaunch(p->graph, p->table->stream));
    MB_CUDA(cudaStreamSynchronize(p->table->stream));
    const double *o = (const double *)(h + 3 * P * 8);
    std::memcpy(val, o, P * 8);
    if (dd) std::memcpy(dd, o + P, P * 8);
    if (dk) std::memcpy(dk, o + 2 * P, P * 8);
    return MB_OK;
}

// ------------------------------------------------------------------ batched Newton polish
//
// Per candidate (search/path1_eval_fast.cpp:103-141 restated on the fused kernel): h0 = K2 at the
// starting delta; then up to `iters` steps delta -= clamp(K2'/K2'', +-max_step) where
// K2' = dK2/ddelta and K2'' = d2K2/ddelta2 = dK2/dk (both returned by the fused kernel); a
// candidate stops moving once |step| < 1e-13 or |K2''| <= 1e-12; finally the larger |h| of the
// start and the end point is kept (with its delta).
namespace {

__global__ void newton_update_kernel(int64_t P, double *delta, const double *dd, const double *dk, double max_step,
                                     unsigned char *done) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P || done[p]) return;
    const double fpp = dk[p];
    if (!(fabs(fpp) > 1e-12)) {
        done[p] = 1;
        return;
    }
    double step = fmin(fmax(dd[p] / fpp, -max_step), max_step);
    delta[p] -= step;
    if (fabs(step) < 1e-13) done[p] = 1;
}

__global__ void newton_choose_kernel(int64_t P, double *delta, const double *delta0, const double *h0, double *val,
                                     double *dd, double *dk, const double *dd0, const double *dk0) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    if (fabs(h0[p]) > fabs(val[p])) {
        val[p] = h0[p];
        delta[p] = delta0[p];
        dd[p] = dd0[p];
        dk[p] = dk0[p];
    }
}

}  // namespace

extern "C" int mb_plan_newton_dev(mb_plan *p, const uint64_t *d_vi, const uint64_t *d_vf, double *d_delta,
                                  int iters, double max_step, double *d_h0, double *d_val, double *d_dd,
                                  double *d_dk, void *stream) {
    MB_CHECK_ARG(p && d_vi && d_vf && d_delta && d_h0 && d_val && d_dd && d_dk, "mb_plan_newton_dev: null argument");
    MB_CHECK_ARG(iters >= 0 && iters <= 1000, "mb_plan_newton_dev: iters=%d", iters);
    MB_CHECK_ARG(std::isfinite(max_step) && max_step > 0, "mb_plan_newton_dev: max_step=%g", max_step);
    MB_TRY(device_guard(p->table->device));
    if (p->P == 0) return MB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t P = (size_t)p->P;
    // plan-owned scratch: delta0, dd0, dk0 and the per-candidate stop flags
    MB_TRY(p->newton_buf.ensure(3 * P * 8 + P + 256));
    double *delta0 = (double *)p->newton_buf.p, *dd0 = delta0 + P, *dk0 = dd0 + P;
    unsigned char *done = (unsigned char *)(dk0 + P);
    const unsigned nb = (unsigned)((P + 255) / 256);
    MB_CUDA(cudaMemcpyAsync(delta0, d_delta, P * 8, cudaMemcpyDeviceToDevice, s));
    MB_CUDA(cudaMemsetAsync(done, 0, P, s));
    MB_TRY(plan_run_dev(p, d_vi, d_vf, d_delta, d_h0, dd0, dk0, s));
    const double *dd_in = dd0, *dk_in = dk0;
    for (int it = 0; it < iters; ++it) {
        newton_update_kernel<<<nb, 256, 0, s>>>(p->P, d_delta, dd_in, dk_in, max_step, done);
        MB_CUDA(cudaGetLastError());
        MB_TRY(plan_run_dev(p, d_vi, d_vf, d_delta, d_val, d_dd, d_dk, s));
        dd_in = d_dd;
        dk_in = d_dk;
    }
    if (iters == 0) {
        MB_CUDA(cudaMemcpyAsync(d_val, d_h0, P * 8, cudaMemcpyDeviceToDevice, s));
        MB_CUDA(cudaMemcpyAsync(d_dd, dd0, P * 8, cudaMemcpyDeviceToDevice, s));
        MB_CUDA(cudaMemcpyAsync(d_dk, dk0, P * 8, cudaMemcpyDeviceToDevice, s));
    }
    newton_choose_kernel<<<nb, 256, 0, s>>>(p->P, d_delta, delta0, d_h0, d_val, d_dd, d_dk, dd0, dk0);
    MB_CUDA(cudaGetLastError());
    return MB_OK;
}

extern "C" int mb_k2_fast(mb_table *h, int64_t P, const uint64_t *v_int, const uint64_t *v_frac,
                          const double *delta, double k, double T, double tol, double *out_val,
                          double *out_dd, double *out_dk, double *err_bound) {
    MB_CHECK_ARG(h && v_int && v_frac && out_val, "mb_k2_fast: null argument");
    mb_plan *p = nullptr;
    MB_TRY(mb_plan_create(h, 1, &P, &k, &T, tol, &p));
    int st = mb_plan_run(p, v_int, v_frac, delta, out_val, out_dd, out_dk);
    if (st == MB_OK && err_bound) *err_bound = p->err_bound[0];
    mb_plan_destroy(p);
    return st;
}
