// Triangle counting: planning units, per-unit features, variant selection
// (forced / heuristic / learned) and the pc_tc entry points.
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "selector.cuh"
#include "tc_kernels.cuh"

namespace pc {
namespace tc {

// ---- planning units ----------------------------------------------------------
// A unit is a run of <= kTile consecutive plist positions inside one
// partition: partitions are the planning granularity, and oversized
// partitions (and the single partition of an unpartitioned graph) are split
// into tiles.

static void build_units(const pc_pgraph* pg, std::vector<int64_t>* lo, std::vector<int64_t>* hi) {
    lo->clear();
    hi->clear();
    for (int k = 0; k < pg->P; ++k) {
        for (int64_t p = pg->pstart[k]; p < pg->pstart[k + 1]; p += kTile) {
            lo->push_back(p);
            hi->push_back(std::min<int64_t>(p + kTile, pg->pstart[k + 1]));
        }
    }
}

// Per-unit raw statistics (one CTA per unit, one warp per pivot).
__global__ void k_unit_stats(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                             const uint32_t* __restrict__ dplus, const int32_t* __restrict__ plist,
                             const int64_t* __restrict__ lo, const int64_t* __restrict__ hi,
                             unsigned long long* __restrict__ out /* kRawStats per unit */) {
    __shared__ unsigned long long s[kRawStats];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    if (tid < kRawStats) s[tid] = 0;
    __syncthreads();
    const int64_t p0 = lo[blockIdx.x], p1 = hi[blockIdx.x];
    unsigned long long npiv = 0, ein = 0, sdp = 0, mdp = 0, mid = 0, sscan = 0, sld = 0, sld2 = 0, s32 = 0;
    for (int64_t p = p0 + warp; p < p1; p += nw) {
        const int32_t b = pivot_at(plist, p);
        const uint64_t rb = off[b], re = off[b + 1];
        const uint32_t dp = dplus[b];
        const uint64_t din = re - rb - dp;
        if (lane == 0) {
            npiv += 1;
            ein += din;
            sdp += dp;
            mdp = max(mdp, (unsigned long long)dp);
            mid = max(mid, (unsigned long long)b + 1);
            const double ld = log2(1.0 + (double)(re - rb));
            sld += (unsigned long long)(ld * 1024.0);
            sld2 += (unsigned long long)(ld * ld * 1024.0);
        }
        if (dp == 0) continue;
        for (uint64_t e = rb + dp + lane; e < re; e += 32) {
            const uint32_t dc = dplus[adj[e]];
            sscan += dc;
            s32 += dc >= 32 ? 1 : 0;
        }
    }
    for (int o = 16; o; o >>= 1) {
        sscan += __shfl_xor_sync(0xffffffffu, sscan, o);
        s32 += __shfl_xor_sync(0xffffffffu, s32, o);
    }
    if (lane == 0) {
        atomicAdd(&s[0], npiv);
        atomicAdd(&s[1], ein);
        atomicAdd(&s[2], sdp);
        atomicMax(&s[3], mdp);
        atomicMax(&s[4], mid);
        atomicAdd(&s[5], sscan);
        atomicAdd(&s[6], sld);
        atomicAdd(&s[7], sld2);
        atomicAdd(&s[8], s32);
    }
    __syncthreads();
    if (tid < kRawStats) out[(uint64_t)blockIdx.x * kRawStats + tid] = s[tid];
}

// Locates linear position q inside a list of position ranges.
__device__ __forceinline__ int64_t range_pos(const int64_t* __restrict__ ranges, const int64_t* __restrict__ rprefix,
                                             uint32_t nranges, uint64_t q) {
    uint32_t lo = 0, hi = nranges;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((uint64_t)rprefix[mid] <= q) lo = mid; else hi = mid;
    }
    return ranges[2 * lo] + (int64_t)(q - (uint64_t)rprefix[lo]);
}

// Work items: per pivot ceil(din / chunk) items; pivots without a set or
// without in-neighbours produce none.
__global__ void k_item_count(const uint64_t* __restrict__ off, const uint32_t* __restrict__ dplus,
                             const int32_t* __restrict__ plist, const int64_t* __restrict__ ranges,
                             const int64_t* __restrict__ rprefix, uint32_t nranges, uint64_t npos, uint32_t chunk,
                             uint32_t* __restrict__ cnt) {
    const uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (q > npos) return;
    if (q == npos) { cnt[q] = 0; return; }
    const int32_t b = pivot_at(plist, range_pos(ranges, rprefix, nranges, q));
    const uint32_t dp = dplus[b];
    const uint64_t din = off[b + 1] - off[b] - dp;
    cnt[q] = (dp == 0 || din == 0) ? 0u : (uint32_t)((din + chunk - 1) / chunk);
}

__global__ void k_item_fill(const int64_t* __restrict__ ranges, const int64_t* __restrict__ rprefix,
                            uint32_t nranges, uint64_t npos, uint32_t chunk, const uint32_t* __restrict__ cnt,
                            const uint32_t* __restrict__ start, Item* __restrict__ items) {
    const uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (q >= npos) return;
    const uint32_t c = cnt[q];
    if (!c) return;
    const int64_t p = range_pos(ranges, rprefix, nranges, q);
    const uint32_t s = start[q];
    for (uint32_t j = 0; j < c; ++j) items[s + j] = Item{(int32_t)p, (int32_t)(j * chunk)};
}

constexpr uint32_t kBitmapCapBits = 1u << 20;  // 128 KB of shared memory

static bool bitmap_feasible(const float* f) { return f[4] <= (float)kBitmapCapBits; }

// Plain autotuned heuristic.  Thresholds come from heuristic_params(), which
// the autotuner (pc_selector_autotune) may replace.
int heuristic_choice(const float* f, const HeuristicParams& hp) {
    const double npiv = f[0], ein = f[1], sdp = f[2], mdp = f[3];
    if (ein <= 0 || sdp <= 0) return -1;
    const double scan = f[5] / std::max(1.0, ein);
    const double inpp = ein / std::max(1.0, npiv);
    if (bitmap_feasible(f) && inpp >= hp.min_in_per_pivot_cta) {
        if (scan >= hp.warp_scan) return PC_VARIANT_BITMAP_WARP;
        if (scan >= hp.group_scan) return PC_VARIANT_BITMAP_GROUP8;
        return PC_VARIANT_BITMAP_LANE;
    }
    if (mdp <= kHashCap) return PC_VARIANT_HASH_WARP;
    if (bitmap_feasible(f)) return PC_VARIANT_BITMAP_GROUP8;
    return PC_VARIANT_MERGE_LANE;
}

bool variant_feasible(int v, const float* f) {
    switch (v) {
        case PC_VARIANT_BITMAP_WARP:
        case PC_VARIANT_BITMAP_GROUP8:
        case PC_VARIANT_BITMAP_LANE: return bitmap_feasible(f);
        default: return v >= 0 && v < PC_NUM_VARIANTS;
    }
}

static uint32_t chunk_of(int v) {
    return (v == PC_VARIANT_BITMAP_WARP || v == PC_VARIANT_BITMAP_GROUP8 || v == PC_VARIANT_BITMAP_LANE)
               ? (uint32_t)kChunkCta
               : (uint32_t)kChunkWarp;
}

}  // namespace tc

using namespace tc;

static pc_status tc_features(pc_pgraph* pg) {
    PC_TRY(ensure_dplus(pg));
    build_units(pg, &pg->unit_lo, &pg->unit_hi);
    const size_t U = pg->unit_lo.size();
    pg->part_features.assign(U * kNumFeatures, 0.f);
    if (U == 0) return PC_OK;
    PC_TRY(scratch_reserve(pg, U * 16 + U * kRawStats * 8));
    int64_t* d_lo = nullptr;
    int64_t* d_hi = nullptr;
    PC_TRY(upload(pg, pg->unit_lo.data(), U, &d_lo));
    PC_TRY(upload(pg, pg->unit_hi.data(), U, &d_hi));
    unsigned long long* d_raw = pg->scratch.take<unsigned long long>(U * kRawStats);
    const int32_t* plist = pg->contiguous ? nullptr : pg->new2old.as<int32_t>();
    k_unit_stats<<<(unsigned)U, 256, 0, pg->g->stream>>>(pg->off, pg->adj, pg->dplus.as<uint32_t>(), plist, d_lo,
                                                        d_hi, d_raw);
    PC_LAUNCHED();
    std::vector<unsigned long long> raw(U * kRawStats);
    PC_CUDA(cudaMemcpyAsync(raw.data(), d_raw, raw.size() * 8, cudaMemcpyDeviceToHost, pg->g->stream));
    PC_TRY(sync(pg));
    for (size_t u = 0; u < U; ++u) raw_to_features(&raw[u * kRawStats], &pg->part_features[u * kNumFeatures]);
    return PC_OK;
}

pc_status tc_ensure_features(pc_pgraph* pg) {
    if (pg->features_ready) return PC_OK;
    PC_TRY(tc_features(pg));
    pg->features_ready = true;
    return PC_OK;
}

// Launches one variant over the given position ranges (all asynchronous).
static pc_status run_variant(pc_pgraph* pg, int v, const std::vector<int64_t>& ranges, uint64_t item_bound,
                             uint32_t max_pivot_plus1, unsigned long long* d_total, uint64_t* launches) {
    cudaStream_t s = pg->g->stream;
    const uint32_t* dp = pg->dplus.as<uint32_t>();
    const int32_t* plist = pg->contiguous ? nullptr : pg->new2old.as<int32_t>();
    const int sms = sm_count(pg->g->device);
    const uint32_t nr = (uint32_t)(ranges.size() / 2);
    std::vector<int64_t> pref(nr + 1, 0);
    for (uint32_t i = 0; i < nr; ++i) pref[i + 1] = pref[i] + (ranges[2 * i + 1] - ranges[2 * i]);
    const uint64_t npos = (uint64_t)pref[nr];
    if (npos == 0) return PC_OK;
    int64_t* d_ranges = nullptr;
    int64_t* d_pref = nullptr;
    PC_TRY(upload(pg, ranges.data(), ranges.size(), &d_ranges));
    PC_TRY(upload(pg, pref.data(), nr + 1, &d_pref));
    const uint32_t chunk = chunk_of(v);
    uint32_t* d_cnt = pg->scratch.take<uint32_t>(npos + 1);
    uint32_t* d_start = pg->scratch.take<uint32_t>(npos + 1);
    size_t tmpb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmpb, d_cnt, d_start, (int64_t)(npos + 1), s);
    void* d_tmp = pg->scratch.take<char>(tmpb);
    uint32_t* d_next = pg->scratch.take<uint32_t>(1);
    Item* d_items = pg->scratch.take<Item>(item_bound);
    if (!d_cnt || !d_start || !d_tmp || !d_next || !d_items)
        return fail(PC_ERR_OOM, "scratch arena too small (internal sizing error)");
    k_item_count<<<(unsigned)ceil_div(npos + 1, 256), 256, 0, s>>>(pg->off, dp, plist, d_ranges, d_pref, nr, npos,
                                                                   chunk, d_cnt);
    PC_LAUNCHED();
    PC_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmpb, d_cnt, d_start, (int64_t)(npos + 1), s));
    count_launch();
    k_item_fill<<<(unsigned)ceil_div(npos, 256), 256, 0, s>>>(d_ranges, d_pref, nr, npos, chunk, d_cnt, d_start,
                                                              d_items);
    PC_LAUNCHED();
    PC_CUDA(cudaMemsetAsync(d_next, 0, 4, s));
    *launches += 3;
    const uint32_t* d_nitems = d_start + npos;
    if (v == PC_VARIANT_BITMAP_WARP || v == PC_VARIANT_BITMAP_GROUP8 || v == PC_VARIANT_BITMAP_LANE) {
        const uint32_t words = (max_pivot_plus1 + 31) / 32;
        const size_t smem = (size_t)words * 4;
        const int ctas_per_sm = smem <= 24 * 1024 ? 4 : (smem <= 48 * 1024 ? 2 : 1);
        const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sms * ctas_per_sm, item_bound));
#define PC_LAUNCH_BM(G)                                                                                        \
    do {                                                                                                       \
        PC_CUDA(cudaFuncSetAttribute(k_tc_bitmap<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
        k_tc_bitmap<G><<<grid, kCtaThreads, smem, s>>>(pg->off, pg->adj, dp, plist, d_items, d_nitems, d_next, \
                                                       d_total, words);                                        \
    } while (0)
        if (v == PC_VARIANT_BITMAP_WARP) PC_LAUNCH_BM(32);
        else if (v == PC_VARIANT_BITMAP_GROUP8) PC_LAUNCH_BM(8);
        else PC_LAUNCH_BM(1);
#undef PC_LAUNCH_BM
    } else {
        const unsigned grid = (unsigned)std::max<uint64_t>(
            1, std::min<uint64_t>((uint64_t)sms * 8, ceil_div(item_bound, kWarpCtaWarps)));
        if (v == PC_VARIANT_HASH_WARP)
            k_tc_warp<kModeHash><<<grid, kWarpCtaWarps * 32, 0, s>>>(pg->off, pg->adj, dp, plist, d_items, d_nitems,
                                                                     d_next, d_total);
        else if (v == PC_VARIANT_MERGE_LANE)
            k_tc_warp<kModeMerge><<<grid, kWarpCtaWarps * 32, 0, s>>>(pg->off, pg->adj, dp, plist, d_items, d_nitems,
                                                                      d_next, d_total);
        else
            k_tc_warp<kModeGallop><<<grid, kWarpCtaWarps * 32, 0, s>>>(pg->off, pg->adj, dp, plist, d_items, d_nitems,
                                                                       d_next, d_total);
    }
    PC_LAUNCHED();
    *launches += 1;
    return PC_OK;
}

// Executes an assignment (one launch group per variant used) and returns the
// count; the only host synchronisation is the final 8-byte read.
static pc_status tc_execute(pc_pgraph* pg, const std::vector<int8_t>& assign, uint64_t* count, pc_tc_stats* stats) {
    cudaStream_t s = pg->g->stream;
    const std::vector<int64_t>& lo = pg->unit_lo;
    const std::vector<int64_t>& hi = pg->unit_hi;
    const std::vector<float>& feat = pg->part_features;
    const size_t U = lo.size();
    struct Group {
        std::vector<int64_t> ranges;
        uint64_t npos = 0, item_bound = 0;
        uint32_t maxid = 0;
    } groups[PC_NUM_VARIANTS];
    for (size_t u = 0; u < U; ++u) {
        const int v = assign[u];
        if (v < 0) continue;
        Group& gr = groups[v];
        if (!gr.ranges.empty() && gr.ranges.back() == lo[u]) gr.ranges.back() = hi[u];
        else { gr.ranges.push_back(lo[u]); gr.ranges.push_back(hi[u]); }
        gr.npos += (uint64_t)(hi[u] - lo[u]);
        // items <= pivots + in-edges / chunk
        gr.item_bound += (uint64_t)(hi[u] - lo[u]) + (uint64_t)(feat[u * kNumFeatures + 1] / chunk_of(v)) + 1;
        gr.maxid = std::max(gr.maxid, (uint32_t)feat[u * kNumFeatures + 4]);
    }
    size_t need = 1024;
    for (int v = 0; v < PC_NUM_VARIANTS; ++v) {
        const Group& gr = groups[v];
        if (gr.ranges.empty()) continue;
        size_t tmpb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tmpb, (uint32_t*)nullptr, (uint32_t*)nullptr, (int64_t)(gr.npos + 1), s);
        need += gr.ranges.size() * 16 + 64 + (gr.npos + 1) * 8 + tmpb + gr.item_bound * sizeof(Item) + 8 * 256;
    }
    PC_TRY(scratch_reserve(pg, need));
    unsigned long long* d_total = pg->scratch.take<unsigned long long>(1);
    uint64_t launches = 0;
    PC_CUDA(cudaEventRecord(pg->ev0, s));
    PC_CUDA(cudaMemsetAsync(d_total, 0, 8, s));
    for (int v = 0; v < PC_NUM_VARIANTS; ++v) {
        const Group& gr = groups[v];
        if (gr.ranges.empty()) continue;
        PC_TRY(run_variant(pg, v, gr.ranges, gr.item_bound, gr.maxid, d_total, &launches));
    }
    PC_CUDA(cudaEventRecord(pg->ev1, s));
    unsigned long long h = 0;
    PC_CUDA(cudaMemcpyAsync(&h, d_total, 8, cudaMemcpyDeviceToHost, s));
    PC_TRY(sync(pg));
    *count = h;
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->partitions = pg->P;
        for (size_t u = 0; u < U; ++u)
            if (assign[u] >= 0) stats->variant_hist[assign[u]]++;
        float ms = 0.f;
        PC_CUDA(cudaEventElapsedTime(&ms, pg->ev0, pg->ev1));
        stats->kernel_ms = ms;
        stats->launches = launches;
        double w = 0;
        for (size_t u = 0; u < U; ++u) w += feat_raw_scan(&feat[u * kNumFeatures]);
        stats->scan_bound = (uint64_t)w;
    }
    return PC_OK;
}

// Chooses a variant per unit.
pc_status tc_assign(pc_pgraph* pg, int32_t variant, const std::vector<float>& feat, size_t U,
                    std::vector<int8_t>* assign, int* selector_used) {
    assign->assign(U, -1);
    if (variant >= 0) {
        if (variant >= PC_NUM_VARIANTS) return fail(PC_ERR_INVALID_INPUT, "unknown TC variant");
        for (size_t u = 0; u < U; ++u) {
            const float* f = &feat[u * kNumFeatures];
            if (f[1] <= 0 || f[2] <= 0) continue;
            if (!variant_feasible(variant, f))
                return fail(PC_ERR_UNSUPPORTED,
                            "forced bitmap variant: a pivot id exceeds the shared-memory bitmap capacity");
            (*assign)[u] = (int8_t)variant;
        }
        *selector_used = 0;
        return PC_OK;
    }
    if (variant != PC_VARIANT_AUTO && variant != PC_VARIANT_HEURISTIC)
        return fail(PC_ERR_INVALID_INPUT, "unknown TC variant");
    const bool learned = (variant == PC_VARIANT_AUTO) && selector_ready(pg->g->device);
    const uint64_t key = selector_version() * 4 + (learned ? 1 : 0);
    if (pg->plan_key == key && pg->plan_assign.size() == U) {
        *assign = pg->plan_assign;
        *selector_used = learned ? 2 : 1;
        return PC_OK;
    }
    const HeuristicParams hp = heuristic_params();
    if (learned) PC_TRY(selector_choose_batch(feat, U, assign));
    for (size_t u = 0; u < U; ++u) {
        const float* f = &feat[u * kNumFeatures];
        if (f[1] <= 0 || f[2] <= 0) { (*assign)[u] = -1; continue; }
        int v = learned ? (*assign)[u] : heuristic_choice(f, hp);
        if (v < 0 || !variant_feasible(v, f)) v = heuristic_choice(f, hp);
        (*assign)[u] = (int8_t)v;
    }
    pg->plan_key = key;
    pg->plan_assign = *assign;
    *selector_used = learned ? 2 : 1;
    return PC_OK;
}

pc_status tc_count(pc_pgraph* pg, int32_t variant, uint64_t* count, pc_tc_stats* stats) {
    PC_TRY(tc_ensure_features(pg));
    const size_t U = pg->unit_lo.size();
    if (U == 0 || pg->g->m == 0) {
        *count = 0;
        if (stats) memset(stats, 0, sizeof(*stats));
        return PC_OK;
    }
    std::vector<int8_t> assign;
    int sel = 0;
    PC_TRY(tc_assign(pg, variant, pg->part_features, U, &assign, &sel));
    PC_TRY(tc_execute(pg, assign, count, stats));
    if (stats) stats->selector = sel;
    return PC_OK;
}

// Times one variant on one unit alone (selector training data).
pc_status tc_time_unit(pc_pgraph* pg, size_t unit, int variant, double* ms, uint64_t* count) {
    PC_TRY(tc_ensure_features(pg));
    const size_t U = pg->unit_lo.size();
    if (unit >= U) return fail(PC_ERR_INVALID_INPUT, "unit index out of range");
    std::vector<int8_t> assign(U, -1);
    assign[unit] = (int8_t)variant;
    pc_tc_stats st;
    PC_TRY(tc_execute(pg, assign, count, &st));
    *ms = st.kernel_ms;
    return PC_OK;
}

}  // namespace pc

using namespace pc;

extern "C" {

pc_status pc_tc_ex(pc_pgraph* pg, int32_t method, int32_t variant, uint64_t* count, pc_tc_stats* stats) {
    clear_error();
    if (!pg || !count) return fail(PC_ERR_INVALID_INPUT, "null argument");
    if (method != PC_METHOD_MERGE && method != PC_METHOD_GALLOPING) return fail(PC_ERR_INVALID_INPUT, "unknown method");
    PC_TRY(use_device(pg->g));
    uint64_t t = 0;
    PC_TRY(tc_count(pg, variant, &t, stats));
    // The galloping form sums |N(u) & N(v)| over every ordered edge (u, v),
    // which counts each triangle 6 times (src/Graph.cpp:1326-1344).
    *count = method == PC_METHOD_MERGE ? t : 6 * t;
    return PC_OK;
}

pc_status pc_tc(pc_pgraph* pg, int32_t method, uint64_t* count) {
    return pc_tc_ex(pg, method, PC_VARIANT_AUTO, count, nullptr);
}

}  // extern "C"
