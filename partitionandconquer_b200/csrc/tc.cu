// Triangle counting: planning units, per-unit features, variant selection
// (forced / heuristic / learned) and the pc_tc entry points.
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <initializer_list>
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

// Unit of every pivot (plist position ranges -> vertex ids).
__global__ void k_unit_of(const int32_t* __restrict__ plist, const int64_t* __restrict__ lo,
                          const int64_t* __restrict__ hi, int32_t* __restrict__ unit_of) {
    const int64_t p0 = lo[blockIdx.x], p1 = hi[blockIdx.x];
    for (int64_t p = p0 + threadIdx.x; p < p1; p += blockDim.x) unit_of[pivot_at(plist, p)] = (int32_t)blockIdx.x;
}

// Per-pivot statistics, one thread per vertex; when a whole warp lies in one
// unit (the common case: units are runs of positions) it reduces first and
// lane 0 issues the atomics.
__global__ void k_unit_pivot_stats(const uint64_t* __restrict__ off, const uint32_t* __restrict__ dplus,
                                   const int32_t* __restrict__ unit_of, uint64_t n,
                                   unsigned long long* __restrict__ out /* kRawStats per unit */) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t nr = (n + 31) & ~31ull;
    const int lane = threadIdx.x & 31;
    for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nr; b += stride) {
        const bool ok = b < n;
        int32_t u = -1;
        unsigned long long v[7] = {0, 0, 0, 0, 0, 0, 0};
        if (ok) {
            u = unit_of[b];
            const uint64_t deg = off[b + 1] - off[b];
            const uint32_t dp = dplus[b];
            const double ld = log2(1.0 + (double)deg);
            v[0] = 1;
            v[1] = deg - dp;
            v[2] = dp;
            v[3] = dp;
            v[4] = b + 1;
            v[5] = (unsigned long long)(ld * 1024.0);
            v[6] = (unsigned long long)(ld * ld * 1024.0);
        }
        const int32_t u0 = __shfl_sync(0xffffffffu, u, 0);
        if (__all_sync(0xffffffffu, ok && u == u0)) {
            for (int o = 16; o; o >>= 1) {
                v[0] += __shfl_xor_sync(0xffffffffu, v[0], o);
                v[1] += __shfl_xor_sync(0xffffffffu, v[1], o);
                v[2] += __shfl_xor_sync(0xffffffffu, v[2], o);
                v[3] = max(v[3], __shfl_xor_sync(0xffffffffu, v[3], o));
                v[4] = max(v[4], __shfl_xor_sync(0xffffffffu, v[4], o));
                v[5] += __shfl_xor_sync(0xffffffffu, v[5], o);
                v[6] += __shfl_xor_sync(0xffffffffu, v[6], o);
            }
            if (lane != 0) continue;
        } else if (!ok) {
            continue;
        }
        unsigned long long* o = out + (uint64_t)u * kRawStats;
        atomicAdd(&o[0], v[0]);
        atomicAdd(&o[1], v[1]);
        atomicAdd(&o[2], v[2]);
        atomicMax(&o[3], v[3]);
        atomicMax(&o[4], v[4]);
        atomicAdd(&o[6], v[5]);
        atomicAdd(&o[7], v[6]);
    }
}

// In-edge statistics: a warp per vertex c streams its prefix N+(c); every
// pivot b there has c as an in-neighbour and gains dplus[c] (the bound on
// c's scan).  Lanes hitting the same unit are merged with __match_any_sync;
// with kSmem (up to kScanStatsSmemUnits units) the per-unit sums gather in a
// shared-memory histogram first, because almost every row starts with hub
// ids and global atomics on the first units would serialise.
constexpr uint32_t kScanStatsSmemUnits = 4096;

template <bool kSmem>
__global__ void k_unit_scan_stats(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                                  const uint32_t* __restrict__ dplus, const int32_t* __restrict__ unit_of,
                                  uint64_t n, uint32_t U, unsigned long long* __restrict__ out) {
    extern __shared__ unsigned long long hist[];  // kSmem: 2 U counters (scan bound, long prefixes)
    if (kSmem) {
        for (uint32_t i = threadIdx.x; i < 2 * U; i += blockDim.x) hist[i] = 0;
        __syncthreads();
    }
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t c = warp; c < n; c += nwarps) {
        const uint32_t dc = dplus[c];
        if (dc == 0) continue;
        const int32_t* row = adj + off[c];
        for (uint32_t k0 = 0; k0 < dc; k0 += 32) {
            const uint32_t k = k0 + lane;
            const bool ok = k < dc;
            const int32_t u = ok ? unit_of[row[k]] : -1;
            const unsigned peers = __match_any_sync(0xffffffffu, u);
            if (ok && lane == __ffs(peers) - 1) {
                const unsigned long long cntp = (unsigned long long)__popc(peers);
                if (kSmem) {
                    atomicAdd(&hist[2 * u], cntp * dc);
                    if (dc >= 32) atomicAdd(&hist[2 * u + 1], cntp);
                } else {
                    atomicAdd(&out[(uint64_t)u * kRawStats + 5], cntp * dc);
                    if (dc >= 32) atomicAdd(&out[(uint64_t)u * kRawStats + 8], cntp);
                }
            }
        }
    }
    if (kSmem) {
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < U; i += blockDim.x) {
            if (hist[2 * i]) atomicAdd(&out[(uint64_t)i * kRawStats + 5], hist[2 * i]);
            if (hist[2 * i + 1]) atomicAdd(&out[(uint64_t)i * kRawStats + 8], hist[2 * i + 1]);
        }
    }
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

// Work items: pivot q (a linear position in the launch's position ranges)
// gives ceil(din / chunk) items, each a run of <= chunk of its in-neighbours;
// pivots without a set or without in-neighbours give none.
__global__ void k_item_count(const uint64_t* __restrict__ off, const uint32_t* __restrict__ dplus,
                             const int32_t* __restrict__ plist, const int64_t* __restrict__ ranges,
                             const int64_t* __restrict__ rprefix, uint32_t nranges, uint64_t npos, uint32_t chunk,
                             uint32_t* __restrict__ cnt) {
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (t > npos) return;
    if (t == npos) { cnt[t] = 0; return; }
    const int32_t b = pivot_at(plist, range_pos(ranges, rprefix, nranges, t));
    const uint32_t dp = dplus[b];
    const uint32_t din = (uint32_t)(off[b + 1] - off[b]) - dp;
    cnt[t] = dp == 0 ? 0u : (din + chunk - 1) / chunk;
}

__global__ void k_item_fill(const uint64_t* __restrict__ off, const uint32_t* __restrict__ dplus,
                            const int32_t* __restrict__ plist, const int64_t* __restrict__ ranges,
                            const int64_t* __restrict__ rprefix, uint32_t nranges, uint64_t npos, uint32_t chunk,
                            const uint32_t* __restrict__ cnt, const uint32_t* __restrict__ start,
                            Item* __restrict__ items, uint32_t cap, uint32_t* __restrict__ nitems) {
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (t == 0) *nitems = min(start[npos], cap);
    if (t >= npos) return;
    const uint32_t c = cnt[t];
    if (!c) return;
    const int64_t p = range_pos(ranges, rprefix, nranges, t);
    const int32_t b = pivot_at(plist, p);
    const uint32_t din = (uint32_t)(off[b + 1] - off[b]) - dplus[b];
    const uint32_t s = start[t];
    for (uint32_t j = 0; j < c && s + j < cap; ++j) {
        const uint32_t j0 = j * chunk;
        items[s + j] = Item{(int32_t)p, (int32_t)j0, (int32_t)min(j0 + chunk, din)};
    }
}

// H[b - lo][a >> 5] |= bit(a) for a in N+(b), one warp per pivot.
__global__ void k_matrix_rows(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                              const uint32_t* __restrict__ dplus, int32_t lo, int32_t hi, uint32_t hstride,
                              uint32_t* __restrict__ H) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t b = lo + warp; b < hi; b += nwarps) {
        const int32_t* row = adj + off[b];
        uint32_t* h = H + (uint64_t)(b - lo) * hstride;
        for (uint32_t k = lane; k < dplus[b]; k += 32) {
            const int32_t a = row[k];
            atomicOr(&h[a >> 5], 1u << (a & 31));
        }
    }
}

// ---- asynchronous staging of an in-neighbour's span into shared memory ----
//
// cp.async (LDGSTS) copies 16-byte pieces global -> shared without passing
// through registers; a lane waits for its own groups (wait_group), and a
// __syncwarp() after the wait makes every lane's pieces visible to the warp.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// A warp-private stage holds up to kStageIds ids of a span (or the smaller
// stage a launch chooses, svec uint4): the copy starts
// at the 16-byte boundary at or below the span (up to 3 ids early) and may
// end up to 3 ids past it, which the 64 ids of padding after the last row
// keep inside the adjacency array.
constexpr uint32_t kStageIds = 256;

// Issues the copies of ids [r, r + k) of adj into stage; returns the offset
// of id r inside it, or -1 when the span does not fit (it is then read from
// global memory).
__device__ __forceinline__ int stage_span(const int32_t* __restrict__ adj, uint64_t r, uint32_t k, uint4* stage,
                                          uint32_t svec, int lane) {
    const uint32_t shift = (uint32_t)(r & 3);
    const uint32_t nvec = (shift + k + 3) >> 2;
    if (nvec > svec) return -1;
    const uint4* src = reinterpret_cast<const uint4*>(adj + (r - shift));
    for (uint32_t x = lane; x < nvec; x += 32) cp_async16(stage + x, src + x);
    return (int)shift;
}

// Word form of a block whose last pivot b sits at position jl: ceil(b/128)
// 16-byte words per row against ceil(jl/32) probe rounds.
__device__ __forceinline__ bool matrix_words_win(int32_t b, uint32_t jl) {
    const uint32_t nv = ((((uint32_t)b + 31) >> 5) + 3) >> 2;
    return ((nv + 31) >> 5) < ((jl + 31) >> 5);
}

// The pairs (b, c) of one in-neighbour c: S = N(c) & [0, min(hi, c)), pivots
// at positions [j0, k).  Pivots are taken U consecutive positions at a time,
// so each step of the warp has U independent row loads in flight per lane and
// shares one load of S (or of its bitmap) between them:
//  - probe form: lanes read S[i] for i below the block's last position and
//    test bit S[i] of each pivot's row (i < j of that pivot);
//  - word form: lanes AND 16-byte words of each row with the warp's
//    shared-memory bitmap of S and count bits.  A row b has bits only below
//    b, so words past a pivot's own length read zeros.
// The form is chosen per block by the rounds each needs; the bitmap is built
// only when some block uses it.  S may point to shared or global memory.
template <int U>
__device__ __forceinline__ unsigned long long matrix_block_pairs(const int32_t* S, uint32_t j0, uint32_t k,
                                                                 int32_t lo, uint32_t hstride,
                                                                 const uint32_t* __restrict__ H, uint32_t* Sb,
                                                                 int lane) {
    unsigned long long cnt = 0;
    bool want = false;
    for (uint32_t jb = j0 + (uint32_t)lane * U; jb < k; jb += 32u * U) {
        const uint32_t jl = min(jb + (uint32_t)U, k) - 1;
        want |= matrix_words_win(S[jl], jl);
    }
    const bool words = __any_sync(0xffffffffu, want);
    if (words) {
        for (uint32_t i = lane; i < k; i += 32) {
            const int32_t a = S[i];
            atomicOr(&Sb[a >> 5], 1u << (a & 31));
        }
        __syncwarp();
    }
    const uint4* Sb4 = reinterpret_cast<const uint4*>(Sb);
    for (uint32_t jb = j0; jb < k; jb += U) {
        const uint32_t ju = min((uint32_t)U, k - jb), jl = jb + ju - 1;
        const int32_t bl = S[jl];
        const uint32_t* h[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int32_t b = (uint32_t)u < ju ? S[jb + u] : bl;
            h[u] = H + (uint64_t)(b - lo) * hstride;
        }
        if (words && matrix_words_win(bl, jl)) {
            const uint32_t nv = ((((uint32_t)bl + 31) >> 5) + 3) >> 2;
            for (uint32_t x = lane; x < nv; x += 32) {
                const uint4 sv = Sb4[x];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if ((uint32_t)u < ju) {
                        const uint4 v = __ldg(reinterpret_cast<const uint4*>(h[u]) + x);
                        cnt += __popc(v.x & sv.x) + __popc(v.y & sv.y) + __popc(v.z & sv.z) + __popc(v.w & sv.w);
                    }
                }
            }
        } else {
            for (uint32_t i = lane; i < jl; i += 32) {
                const int32_t a = S[i];
                const uint32_t w = (uint32_t)a >> 5, bit = (uint32_t)a & 31;
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if ((uint32_t)u < ju && i < jb + (uint32_t)u) cnt += (__ldg(h[u] + w) >> bit) & 1u;
            }
        }
    }
    if (words) {
        __syncwarp();
        for (uint32_t i = lane; i < k; i += 32) Sb[S[i] >> 5] = 0;
        __syncwarp();
    }
    return cnt;
}

// Pivot positions [klo, khi) of in-neighbour c in its row (N(c) is sorted,
// and min(hi, c) <= c keeps the search inside N+(c)).
__device__ __forceinline__ void matrix_span(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                                            const uint32_t* __restrict__ dplus, int32_t lo, int32_t hi, uint64_t c,
                                            uint64_t* r, uint32_t* klo, uint32_t* khi) {
    *r = off[c];
    const int32_t lim = (int64_t)c < (int64_t)hi ? (int32_t)c : hi;
    *khi = lower_bound_i32(adj + *r, dplus[c], lim);
    *klo = lower_bound_i32(adj + *r, *khi, lo);
}

// In-neighbours c run in two phases.  The first kMatrixHeavy ids after lo
// (the hubs, with the longest S_c) are taken one per warp from counter
// next[0], their spans read from global memory; the rest 32 at a time from
// next[1], lanes locating the 32 spans at once.  In the second phase the
// spans are staged into two warp-private shared-memory buffers by cp.async:
// the next span's copies are in flight while the current one is counted.
// One-at-a-time for the hubs keeps a single warp from holding a batch of 32
// hubs at the end of the launch.
constexpr uint64_t kMatrixHeavy = 65536;

template <int U>
__global__ void __launch_bounds__(kMatrixWarps * 32) k_tc_matrix(const uint64_t* __restrict__ off,
                                                               const int32_t* __restrict__ adj,
                                                               const uint32_t* __restrict__ dplus, int32_t lo,
                                                               int32_t hi, uint64_t n, uint32_t hstride,
                                                               const uint32_t* __restrict__ H,
                                                               unsigned long long* __restrict__ next,
                                                               unsigned long long* __restrict__ total,
                                                               unsigned long long* __restrict__ unit_cost,
                                                               int32_t unit, uint32_t svec) {
    extern __shared__ uint4 msm4[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t nwarps = blockDim.x >> 5;  // kMatrixWarps or fewer
    uint32_t* Sb = reinterpret_cast<uint32_t*>(msm4) + (size_t)w * hstride;  // warp-private bitmap of S_c
    uint4* stage = msm4 + (size_t)nwarps * (hstride / 4) + (size_t)w * 2 * svec;
    for (uint32_t i = lane; i < hstride; i += 32) Sb[i] = 0;
    __syncwarp();
    const long long t0 = unit_cost ? clock64() : 0;
    unsigned long long cnt = 0;
    const uint64_t c1 = (uint64_t)lo + 1 + kMatrixHeavy < n ? (uint64_t)lo + 1 + kMatrixHeavy : n;
    for (;;) {  // phase 1: one hub in-neighbour per grab
        unsigned long long q = 0;
        if (lane == 0) q = atomicAdd(&next[0], 1ull);
        const uint64_t c = __shfl_sync(0xffffffffu, q, 0) + (uint64_t)lo + 1;
        if (c >= c1) break;
        uint64_t r = 0;
        uint32_t klo = 0, khi = 0;
        if (lane == 0) matrix_span(off, adj, dplus, lo, hi, c, &r, &klo, &khi);
        r = __shfl_sync(0xffffffffu, r, 0);
        klo = __shfl_sync(0xffffffffu, klo, 0);
        khi = __shfl_sync(0xffffffffu, khi, 0);
        if (khi > klo) cnt += matrix_block_pairs<U>(adj + r, klo, khi, lo, hstride, H, Sb, lane);
    }
    for (;;) {  // phase 2: 32 in-neighbours per grab, spans staged two deep
        unsigned long long q = 0;
        if (lane == 0) q = atomicAdd(&next[1], 32ull);
        const uint64_t base = __shfl_sync(0xffffffffu, q, 0) + c1;
        if (base >= n) break;
        const uint64_t c = base + lane;
        uint64_t r = 0;
        uint32_t klo = 0, khi = 0;
        if (c < n) matrix_span(off, adj, dplus, lo, hi, c, &r, &klo, &khi);
        unsigned todo = __ballot_sync(0xffffffffu, khi > klo);
        if (!todo) continue;
        int src = __ffs(todo) - 1;
        todo &= todo - 1;
        int buf = 0;
        int shift = stage_span(adj, __shfl_sync(0xffffffffu, r, src), __shfl_sync(0xffffffffu, khi, src),
                               stage, svec, lane);
        cp_async_commit();
        for (;;) {
            const int nxt = todo ? __ffs(todo) - 1 : -1;
            if (nxt >= 0) todo &= todo - 1;
            int nshift = -1;
            if (nxt >= 0)
                nshift = stage_span(adj, __shfl_sync(0xffffffffu, r, nxt), __shfl_sync(0xffffffffu, khi, nxt),
                                    stage + (buf ^ 1) * svec, svec, lane);
            cp_async_commit();
            cp_async_wait<1>();  // every group but the one just issued: the current span is in place
            __syncwarp();
            const uint64_t rs = __shfl_sync(0xffffffffu, r, src);
            const uint32_t j0 = __shfl_sync(0xffffffffu, klo, src);
            const uint32_t k = __shfl_sync(0xffffffffu, khi, src);
            const int32_t* S = shift >= 0 ? reinterpret_cast<const int32_t*>(stage + buf * svec) + shift
                                          : adj + rs;
            cnt += matrix_block_pairs<U>(S, j0, k, lo, hstride, H, Sb, lane);
            __syncwarp();  // the buffer just read is the next stage's target
            if (nxt < 0) break;
            src = nxt;
            shift = nshift;
            buf ^= 1;
        }
    }
    cp_async_wait<0>();
    if (unit_cost) {
        __syncwarp();
        if (lane == 0) atomicAdd(&unit_cost[unit], (unsigned long long)(clock64() - t0));
    }
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0 && cnt) atomicAdd(total, cnt);
}

constexpr uint32_t kBitmapCapBits = 1u << 20;  // 128 KB of shared memory

static bool bitmap_feasible(const float* f) { return f[4] <= (float)kBitmapCapBits; }
// The in-neighbour-major form needs the unit's pivots to be the id range
// [lo, hi) (contiguous partitions; tc_assign checks that) with hi <= 2^16,
// and its resident rows to fit L2 (126 MB on B200): rows that spill re-read
// DRAM on every probe, which is what the form exists to avoid (RMAT-24's
// fourth hub unit, 128 MB of rows, cost 4 ms more than the bitmap kernel).
constexpr double kMatrixRowsCap = 100.0 * (1 << 20);
static bool matrix_feasible(const float* f) {
    const double words = (double)((((uint64_t)f[4] + 31) / 32 + 3) & ~(uint64_t)3);
    return f[4] <= (float)kMatrixMaxId && (double)f[0] * words * 4.0 <= kMatrixRowsCap;
}

// Plain autotuned heuristic.  Thresholds come from heuristic_params(), which
// the autotuner (pc_selector_autotune) may replace.
int heuristic_choice(const float* f, const HeuristicParams& hp) {
    const double npiv = f[0], ein = f[1], sdp = f[2], mdp = f[3];
    if (ein <= 0 || sdp <= 0) return -1;
    const double scan = f[5] / std::max(1.0, ein);
    const double inpp = ein / std::max(1.0, npiv);
    if (matrix_feasible(f) && inpp >= hp.min_in_per_pivot_cta && scan >= hp.matrix_scan) return PC_VARIANT_MATRIX;
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
        case PC_VARIANT_MATRIX: return matrix_feasible(f);
        default: return v >= 0 && v < PC_NUM_VARIANTS;
    }
}

static bool is_bitmap(int v) {
    return v == PC_VARIANT_BITMAP_WARP || v == PC_VARIANT_BITMAP_GROUP8 || v == PC_VARIANT_BITMAP_LANE;
}

// Bitmap sets per CTA: K warps share one set; the smallest K whose 16/K sets
// fit the shared-memory budget (about 100 KB for two CTAs per SM, up to
// 200 KB for one).
struct BitmapShape {
    int K;
    uint32_t words;
    size_t smem;
    int ctas_per_sm;
};

static BitmapShape bitmap_shape(uint32_t max_pivot_plus1) {
    BitmapShape sh{};
    sh.words = std::max<uint32_t>(1, (max_pivot_plus1 + 31) / 32);
    const size_t budget_two = 100 * 1024, budget_one = 200 * 1024;
    for (int K = 1; K <= 16; K *= 2) {
        const size_t smem = (size_t)(16 / K) * sh.words * 4;
        if (smem <= budget_two || (K == 16 && smem <= budget_one)) {
            sh.K = K;
            sh.smem = smem;
            break;
        }
    }
    if (!sh.K) {
        sh.K = 16;
        sh.smem = (size_t)sh.words * 4;
    }
    sh.ctas_per_sm = (int)std::max<size_t>(1, std::min<size_t>(4, (220 * 1024) / (sh.smem + 1024)));
    return sh;
}

// Arguments of one bitmap-kernel launch.
struct BitmapLaunch {
    unsigned grid;
    size_t smem;
    cudaStream_t s;
    const uint64_t* off;
    const int32_t* adj;
    const uint32_t* dp;
    const int32_t* plist;
    const Item* items;
    const uint32_t* nitems;
    uint32_t* next;
    unsigned long long* total;
    uint32_t words;
    unsigned long long* cost;
    const int32_t* unit_of;
    unsigned long long* tri;  // per-vertex triangle counts (LCC), or null
    uint32_t* ecnt;           // per-edge counts at the oriented slots (Jaccard), or null
};

template <int K, int G, bool kVC, bool kEC, bool kSplit = false>
static pc_status launch_bitmap_kgv(const BitmapLaunch& L) {
    PC_CUDA(cudaFuncSetAttribute(k_tc_bitmap<K, G, kVC, kEC, kSplit>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)L.smem));
    k_tc_bitmap<K, G, kVC, kEC, kSplit><<<L.grid, kCtaThreads, L.smem, L.s>>>(
        L.off, L.adj, L.dp, L.plist, L.items, L.nitems, L.next, L.total, L.words, L.cost, L.unit_of, L.tri, L.ecnt);
    return PC_OK;
}

// Split-set launches: sets of kSplitWords + kHashSlots words (10 KB); K = 2
// in the count mode (16 sets per SM), K = 4 in the per-vertex mode, whose
// 32 KB hub histogram per CTA would leave one CTA of 8 sets per SM.
static pc_status launch_bitmap_split(int K, int G, const BitmapLaunch& L) {
    if (L.ecnt || (L.tri ? K != 4 : K != 2)) return fail(PC_ERR_UNSUPPORTED, "split pivot sets: unexpected launch shape");
    if (L.tri) {
        if (G == 32) return launch_bitmap_kgv<4, 32, true, false, true>(L);
        if (G == 8) return launch_bitmap_kgv<4, 8, true, false, true>(L);
        return launch_bitmap_kgv<4, 1, true, false, true>(L);
    }
    if (G == 32) return launch_bitmap_kgv<2, 32, false, false, true>(L);
    if (G == 8) return launch_bitmap_kgv<2, 8, false, false, true>(L);
    return launch_bitmap_kgv<2, 1, false, false, true>(L);
}

template <int K, bool kVC, bool kEC>
static pc_status launch_bitmap_kmode(int G, const BitmapLaunch& L) {
    if (G == 32) return launch_bitmap_kgv<K, 32, kVC, kEC>(L);
    if (G == 8) return launch_bitmap_kgv<K, 8, kVC, kEC>(L);
    return launch_bitmap_kgv<K, 1, kVC, kEC>(L);
}

template <int K>
static pc_status launch_bitmap_k(int G, const BitmapLaunch& L) {
    if (L.tri) return launch_bitmap_kmode<K, true, false>(G, L);
    if (L.ecnt) return launch_bitmap_kmode<K, false, true>(G, L);
    return launch_bitmap_kmode<K, false, false>(G, L);
}

static pc_status launch_bitmap(int K, int G, const BitmapLaunch& L) {
    switch (K) {
        case 1: return launch_bitmap_k<1>(G, L);
        case 2: return launch_bitmap_k<2>(G, L);
        case 4: return launch_bitmap_k<4>(G, L);
        case 8: return launch_bitmap_k<8>(G, L);
        default: return launch_bitmap_k<16>(G, L);
    }
}


}  // namespace tc

using namespace tc;

static pc_status tc_features(pc_pgraph* pg) {
    PC_TRY(ensure_dplus(pg));
    build_units(pg, &pg->unit_lo, &pg->unit_hi);
    const size_t U = pg->unit_lo.size();
    const uint64_t n = pg->g->n;
    pg->part_features.assign(U * kNumFeatures, 0.f);
    if (U == 0) return PC_OK;
    PC_TRY(pg->unit_of.ensure(std::max<uint64_t>(n, 1) * 4, "unit of vertex"));
    PC_TRY(scratch_reserve(pg, U * 16 + U * kRawStats * 8));
    int64_t* d_lo = nullptr;
    int64_t* d_hi = nullptr;
    PC_TRY(upload(pg, pg->unit_lo.data(), U, &d_lo));
    PC_TRY(upload(pg, pg->unit_hi.data(), U, &d_hi));
    unsigned long long* d_raw = pg->scratch.take<unsigned long long>(U * kRawStats);
    cudaStream_t s = pg->g->stream;
    PC_CUDA(cudaMemsetAsync(d_raw, 0, U * kRawStats * 8, s));
    const int32_t* plist = pg->contiguous ? nullptr : pg->new2old.as<int32_t>();
    int32_t* unit_of = pg->unit_of.as<int32_t>();
    const int sms = sm_count(pg->g->device);
    k_unit_of<<<(unsigned)U, 256, 0, s>>>(plist, d_lo, d_hi, unit_of);
    PC_LAUNCHED();
    k_unit_pivot_stats<<<sms * 8, 256, 0, s>>>(pg->off, pg->dplus.as<uint32_t>(), unit_of, n, d_raw);
    PC_LAUNCHED();
    if (U <= kScanStatsSmemUnits) {
        const size_t smem = 2 * U * sizeof(unsigned long long);
        PC_CUDA(cudaFuncSetAttribute(k_unit_scan_stats<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_unit_scan_stats<true><<<sms * 2, 1024, smem, s>>>(pg->off, pg->adj, pg->dplus.as<uint32_t>(), unit_of, n,
                                                           (uint32_t)U, d_raw);
    } else {
        k_unit_scan_stats<false><<<sms * 16, 256, 0, s>>>(pg->off, pg->adj, pg->dplus.as<uint32_t>(), unit_of, n,
                                                           (uint32_t)U, d_raw);
    }
    PC_LAUNCHED();
    std::vector<unsigned long long> raw(U * kRawStats);
    PC_CUDA(cudaMemcpyAsync(raw.data(), d_raw, raw.size() * 8, cudaMemcpyDeviceToHost, s));
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

// One launch: a variant and its bitmap shape (words rounded up to a power
// of two).
struct LaunchGroup {
    int v = -1;
    uint32_t words = 0;
    bool split = false;  // bitmap variants: SplitSets (kSplitWords bitmap words + a hash)
    std::vector<int64_t> ranges;
    uint64_t npos = 0, item_bound = 0;
    double ein = 0;
    size_t units = 0;
    std::vector<int32_t> unit_ids;  // matrix groups: one launch per unit (ranges not merged)
};

// Words per resident pivot bitmap row of a matrix unit with ids below hi:
// ceil(hi / 32) rounded up to 16 bytes, so rows can be read as uint4.
static uint32_t matrix_stride(int64_t hi) { return (uint32_t)((((hi + 31) / 32) + 3) & ~(int64_t)3); }

// Bytes of the resident pivot bitmap rows of a matrix unit [lo, hi).
static uint64_t matrix_bytes(int64_t lo, int64_t hi) { return (uint64_t)(hi - lo) * matrix_stride(hi) * 4; }

// Bitmap units whose pivot ids reach kSplitLo or more run with SplitSets in
// the count and per-vertex modes, unless PC_BITMAP_SPLIT=0 is in the
// environment (read once; a switch for measurements).
static bool bitmap_split_enabled() {
    static const bool on = [] {
        const char* e = getenv("PC_BITMAP_SPLIT");
        return !(e && atoi(e) == 0);
    }();
    return on;
}

// Pivots per block of the matrix kernel: 4, or 8 with PC_MATRIX_PIVOT_BLOCK=8
// in the environment (read once; a tuning override for measurements).
static int matrix_pivot_block() {
    static const int u = [] {
        const char* e = getenv("PC_MATRIX_PIVOT_BLOCK");
        return (e && atoi(e) == 8) ? 8 : 4;
    }();
    return u;
}

// Matrix launch shape: warps per CTA (kMatrixWarps, or PC_MATRIX_WARPS=4) and
// ids per span stage (kStageIds, or PC_MATRIX_STAGE_IDS=128|512|1024), read
// once from the environment; switches for measurements.
static int matrix_env(const char* name, int dflt, std::initializer_list<int> allowed) {
    const char* e = getenv(name);
    if (!e) return dflt;
    const int v = atoi(e);
    for (int a : allowed)
        if (a == v) return v;
    return dflt;
}
static int matrix_warps() {
    static const int w = matrix_env("PC_MATRIX_WARPS", kMatrixWarps, {4, 8});
    return w;
}
static uint32_t matrix_stage_vec() {
    static const uint32_t v = (uint32_t)matrix_env("PC_MATRIX_STAGE_IDS", (int)kStageIds, {128, 256, 512, 1024}) / 4 + 1;
    return v;
}

template <int U>
static pc_status launch_matrix(pc_pgraph* pg, int64_t lo, int64_t hi, uint32_t hstride, const uint32_t* H,
                               unsigned long long* d_next, unsigned long long* d_total, unsigned long long* d_cost,
                               int32_t unit, int sms, cudaStream_t s) {
    const int warps = matrix_warps();
    const uint32_t svec = matrix_stage_vec();
    const size_t smem = (size_t)warps * hstride * 4 + (size_t)warps * 2 * svec * sizeof(uint4);
    PC_CUDA(cudaFuncSetAttribute(k_tc_matrix<U>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    PC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tc_matrix<U>, warps * 32, smem));
    k_tc_matrix<U><<<(unsigned)(sms * std::max(1, per_sm)), warps * 32, smem, s>>>(
        pg->off, pg->adj, pg->dplus.as<uint32_t>(), (int32_t)lo, (int32_t)hi, pg->g->n, hstride, H, d_next, d_total,
        d_cost, unit, svec);
    PC_LAUNCHED();
    return PC_OK;
}

// The in-neighbour-major form over one unit (ids [lo, hi)), all asynchronous:
// rows H built from N+(b), then the walk over the in-neighbours.
static pc_status run_matrix_unit(pc_pgraph* pg, int64_t lo, int64_t hi, int32_t unit, uint32_t* H,
                                 unsigned long long* d_next, unsigned long long* d_total, unsigned long long* d_cost,
                                 uint64_t* launches) {
    cudaStream_t s = pg->g->stream;
    const int sms = sm_count(pg->g->device);
    const uint32_t hstride = matrix_stride(hi);
    PC_CUDA(cudaMemsetAsync(H, 0, matrix_bytes(lo, hi), s));
    PC_CUDA(cudaMemsetAsync(d_next, 0, 16, s));
    k_matrix_rows<<<sms * 8, 256, 0, s>>>(pg->off, pg->adj, pg->dplus.as<uint32_t>(), (int32_t)lo, (int32_t)hi, hstride,
                                          H);
    PC_LAUNCHED();
    if (matrix_pivot_block() == 8)
        PC_TRY(launch_matrix<8>(pg, lo, hi, hstride, H, d_next, d_total, d_cost, unit, sms, s));
    else
        PC_TRY(launch_matrix<4>(pg, lo, hi, hstride, H, d_next, d_total, d_cost, unit, sms, s));
    *launches += 2;
    return PC_OK;
}

// Items never exceed min(pivots, in-edges) + in-edges / chunk; the float
// in-edge feature is widened by 256 per unit for its rounding.
static void finish_group(LaunchGroup* gr) {
    const uint64_t ein = (uint64_t)gr->ein + 256 * gr->units;
    gr->item_bound = std::min<uint64_t>(gr->npos, ein) + ein / 256 + 1;
}

// Launches one group (all asynchronous).
static pc_status run_group(pc_pgraph* pg, const LaunchGroup& gr, unsigned long long* d_total, uint64_t* launches,
                           unsigned long long* d_cost, unsigned long long* d_tri, uint32_t* d_ecnt) {
    if (gr.v == PC_VARIANT_MATRIX) {
        uint64_t hb = 0;
        for (size_t i = 0; i < gr.unit_ids.size(); ++i) hb = std::max(hb, matrix_bytes(gr.ranges[2 * i], gr.ranges[2 * i + 1]));
        uint32_t* H = pg->scratch.take<uint32_t>(hb / 4);
        unsigned long long* d_next = pg->scratch.take<unsigned long long>(2);
        if (!H || !d_next) return fail(PC_ERR_OOM, "scratch arena too small (internal sizing error)");
        for (size_t i = 0; i < gr.unit_ids.size(); ++i)
            PC_TRY(run_matrix_unit(pg, gr.ranges[2 * i], gr.ranges[2 * i + 1], gr.unit_ids[i], H, d_next, d_total,
                                   d_cost, launches));
        return PC_OK;
    }
    const int32_t* unit_of = pg->unit_of.as<int32_t>();
    cudaStream_t s = pg->g->stream;
    const int v = gr.v;
    const uint32_t* dp = pg->dplus.as<uint32_t>();
    const int32_t* plist = pg->contiguous ? nullptr : pg->new2old.as<int32_t>();
    const int sms = sm_count(pg->g->device);
    const uint32_t nr = (uint32_t)(gr.ranges.size() / 2);
    std::vector<int64_t> pref(nr + 1, 0);
    for (uint32_t i = 0; i < nr; ++i) pref[i + 1] = pref[i] + (gr.ranges[2 * i + 1] - gr.ranges[2 * i]);
    const uint64_t npos = (uint64_t)pref[nr];
    if (npos == 0) return PC_OK;
    int64_t* d_ranges = nullptr;
    int64_t* d_pref = nullptr;
    PC_TRY(upload(pg, gr.ranges.data(), gr.ranges.size(), &d_ranges));
    PC_TRY(upload(pg, pref.data(), nr + 1, &d_pref));
    BitmapShape sh = bitmap_shape((gr.split ? kSplitWords + (uint32_t)kHashSlots : gr.words) * 32u);
    if (gr.split && d_tri) {
        sh.K = 4;
        sh.smem = (size_t)(16 / sh.K) * (kSplitWords + kHashSlots) * 4;
    }
    const uint32_t chunk = is_bitmap(v) ? 256u * (uint32_t)sh.K : (uint32_t)kChunkWarp;
    uint32_t* d_cnt = pg->scratch.take<uint32_t>(npos + 1);
    uint32_t* d_start = pg->scratch.take<uint32_t>(npos + 1);
    size_t tmpb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmpb, d_cnt, d_start, (int64_t)(npos + 1), s);
    void* d_tmp = pg->scratch.take<char>(tmpb);
    uint32_t* d_next = pg->scratch.take<uint32_t>(2);
    Item* d_items = pg->scratch.take<Item>(gr.item_bound);
    if (!d_cnt || !d_start || !d_tmp || !d_next || !d_items)
        return fail(PC_ERR_OOM, "scratch arena too small (internal sizing error)");
    k_item_count<<<(unsigned)ceil_div(npos + 1, 256), 256, 0, s>>>(pg->off, dp, plist, d_ranges, d_pref, nr, npos,
                                                                   chunk, d_cnt);
    PC_LAUNCHED();
    PC_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmpb, d_cnt, d_start, (int64_t)(npos + 1), s));
    count_launch();
    k_item_fill<<<(unsigned)ceil_div(npos, 256), 256, 0, s>>>(pg->off, dp, plist, d_ranges, d_pref, nr, npos, chunk,
                                                              d_cnt, d_start, d_items, (uint32_t)gr.item_bound,
                                                              d_next + 1);
    PC_LAUNCHED();
    PC_CUDA(cudaMemsetAsync(d_next, 0, 4, s));
    *launches += 3;
    const uint32_t* d_nitems = d_next + 1;
    if (is_bitmap(v)) {
        BitmapLaunch L;
        const size_t nsets = (size_t)(kCtaThreads / 32 / sh.K);
        L.smem = sh.smem + (d_tri ? (size_t)kHubHist * 4 : 0) +
                 (d_ecnt ? nsets * (((sh.words + 7) / 8) + (size_t)kEcRankCap) * 4 : 0);
        const int cps = (d_tri || d_ecnt)
                            ? (int)std::max<size_t>(1, std::min<size_t>(4, (220 * 1024) / (L.smem + 1024)))
                            : sh.ctas_per_sm;
        L.grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sms * cps, gr.item_bound));
        L.s = s;
        L.off = pg->off;
        L.adj = pg->adj;
        L.dp = dp;
        L.plist = plist;
        L.items = d_items;
        L.nitems = d_nitems;
        L.next = d_next;
        L.total = d_total;
        L.words = gr.split ? kSplitWords : sh.words;
        L.cost = d_cost;
        L.unit_of = unit_of;
        L.tri = d_tri;
        L.ecnt = d_ecnt;
        const int Gsel = v == PC_VARIANT_BITMAP_WARP ? 32 : (v == PC_VARIANT_BITMAP_GROUP8 ? 8 : 1);
        if (gr.split) PC_TRY(launch_bitmap_split(sh.K, Gsel, L));
        else PC_TRY(launch_bitmap(sh.K, Gsel, L));
    } else {
        const unsigned grid = (unsigned)std::max<uint64_t>(
            1, std::min<uint64_t>((uint64_t)sms * 8, ceil_div(gr.item_bound, kWarpCtaWarps)));
        const unsigned bs = kWarpCtaWarps * 32;
        if (d_ecnt) {
            if (v == PC_VARIANT_HASH_WARP)
                k_tc_warp<kModeHash, false, true><<<grid, bs, 0, s>>>(pg->off, pg->adj, dp, plist, d_items, d_nitems,
                                                                      d_next, d_total, d_cost, unit_of, nullptr, d_ecnt);
            else if (v == PC_VARIANT_MERGE_LANE)
                k_tc_warp<kModeMerge, false, true><<<grid, bs, 0, s>>>(pg->off, pg->adj, dp, plist, d_items, d_nitems,
                                                                       d_next, d_total, d_cost, unit_of, nullptr,
                                                                       d_ecnt);
            else
                k_tc_warp<kModeGallop, false, true><<<grid, bs, 0, s>>>(pg->off, pg->adj, dp, plist, d_items,
                                                                        d_nitems, d_next, d_total, d_cost, unit_of,
                                                                        nullptr, d_ecnt);
        } else if (d_tri) {
            if (v == PC_VARIANT_HASH_WARP)
                k_tc_warp<kModeHash, true><<<grid, bs, 0, s>>>(pg->off, pg->adj, dp, plist, d_items, d_nitems, d_next,
                                                               d_total, d_cost, unit_of, d_tri);
            else if (v == PC_VARIANT_MERGE_LANE)
                k_tc_warp<kModeMerge, true><<<grid, bs, 0, s>>>(pg->off, pg->adj, dp, plist, d_items, d_nitems, d_next,
                                                                d_total, d_cost, unit_of, d_tri);
            else
                k_tc_warp<kModeGallop, true><<<grid, bs, 0, s>>>(pg->off, pg->adj, dp, plist, d_items, d_nitems,
                                                                 d_next, d_total, d_cost, unit_of, d_tri);
        } else if (v == PC_VARIANT_HASH_WARP) {
            k_tc_warp<kModeHash><<<grid, bs, 0, s>>>(pg->off, pg->adj, dp, plist, d_items, d_nitems, d_next, d_total,
                                                     d_cost, unit_of);
        } else if (v == PC_VARIANT_MERGE_LANE) {
            k_tc_warp<kModeMerge><<<grid, bs, 0, s>>>(pg->off, pg->adj, dp, plist, d_items, d_nitems, d_next, d_total,
                                                      d_cost, unit_of);
        } else {
            k_tc_warp<kModeGallop><<<grid, bs, 0, s>>>(pg->off, pg->adj, dp, plist, d_items, d_nitems, d_next, d_total,
                                                       d_cost, unit_of);
        }
    }
    PC_LAUNCHED();
    *launches += 1;
    return PC_OK;
}

// Executes an assignment (one launch group per variant and bitmap shape
// used) and returns the count; the only host synchronisation is the final
// 8-byte read.  With unit_ms (profiling runs) the kernels also charge their
// warp-cycles to the units, every group is timed by its own events, and each
// unit gets its group's time in proportion to its cycles: the unit's cost
// inside a full run, where it shares the GPU with the other units.
static pc_status tc_execute(pc_pgraph* pg, const std::vector<int8_t>& assign, uint64_t* count, pc_tc_stats* stats,
                            std::vector<double>* unit_ms = nullptr, unsigned long long* d_tri = nullptr,
                            uint32_t* d_ecnt = nullptr) {
    cudaStream_t s = pg->g->stream;
    const std::vector<int64_t>& lo = pg->unit_lo;
    const std::vector<int64_t>& hi = pg->unit_hi;
    const std::vector<float>& feat = pg->part_features;
    const size_t U = lo.size();
    // Bitmap units are grouped by their bitmap size rounded up to a power of
    // two, so the hub units (small ids) get small sets and more CTAs per SM;
    // in the count and per-vertex modes, units with pivot ids past kSplitLo
    // share one group of fixed-size SplitSets (class kClasses).
    constexpr int kClasses = 16;
    const bool split_ok = bitmap_split_enabled() && !d_ecnt;
    std::vector<LaunchGroup> groups(PC_NUM_VARIANTS * (kClasses + 1));
    std::vector<int> group_of(U, -1);
    for (size_t u = 0; u < U; ++u) {
        const int v = assign[u];
        if (v < 0) continue;
        const uint32_t mid = (uint32_t)feat[u * kNumFeatures + 4];
        int c = 0;
        if (is_bitmap(v)) {
            const uint32_t w = std::max<uint32_t>(1, (mid + 31) / 32);
            while ((1u << c) < w && c < kClasses - 1) ++c;
            if (split_ok && mid > (uint32_t)kSplitLo) c = kClasses;
        }
        LaunchGroup& gr = groups[v * (kClasses + 1) + c];
        group_of[u] = v * (kClasses + 1) + c;
        gr.v = v;
        gr.split = c == kClasses;
        gr.words = gr.split ? kSplitWords : 1u << c;
        if (v == PC_VARIANT_MATRIX) {
            gr.ranges.push_back(lo[u]);
            gr.ranges.push_back(hi[u]);
            gr.unit_ids.push_back((int32_t)u);
        } else if (!gr.ranges.empty() && gr.ranges.back() == lo[u]) {
            gr.ranges.back() = hi[u];
        } else {
            gr.ranges.push_back(lo[u]);
            gr.ranges.push_back(hi[u]);
        }
        gr.npos += (uint64_t)(hi[u] - lo[u]);
        gr.ein += feat[u * kNumFeatures + 1];
        gr.units += 1;
    }
    size_t need = 1024;
    for (LaunchGroup& gr : groups) {
        if (gr.ranges.empty()) continue;
        if (gr.v == PC_VARIANT_MATRIX) {
            uint64_t hb = 0;
            for (size_t i = 0; i < gr.unit_ids.size(); ++i)
                hb = std::max(hb, matrix_bytes(gr.ranges[2 * i], gr.ranges[2 * i + 1]));
            need += hb + 2 * 256;
            continue;
        }
        finish_group(&gr);
        size_t tmpb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tmpb, (uint32_t*)nullptr, (uint32_t*)nullptr, (int64_t)(gr.npos + 1),
                                      s);
        need += gr.ranges.size() * 16 + 64 + (gr.npos + 1) * 8 + tmpb + gr.item_bound * sizeof(Item) + 8 * 256;
    }
    if (unit_ms) need += U * 8 + 256;
    PC_TRY(scratch_reserve(pg, need));
    unsigned long long* d_total = pg->scratch.take<unsigned long long>(1);
    unsigned long long* d_cost = unit_ms ? pg->scratch.take<unsigned long long>(std::max<size_t>(U, 1)) : nullptr;
    std::vector<cudaEvent_t> gev;
    auto drop_events = [&]() {
        for (cudaEvent_t e : gev) cudaEventDestroy(e);
        gev.clear();
    };
    if (unit_ms) {
        gev.resize(2 * groups.size(), nullptr);
        for (cudaEvent_t& e : gev)
            if (cudaEventCreate(&e) != cudaSuccess) {
                drop_events();
                return fail(PC_ERR_CUDA, "event creation failed");
            }
        PC_CUDA(cudaMemsetAsync(d_cost, 0, std::max<size_t>(U, 1) * 8, s));
    }
    uint64_t launches = 0;
    PC_CUDA(cudaEventRecord(pg->ev0, s));
    PC_CUDA(cudaMemsetAsync(d_total, 0, 8, s));
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        const LaunchGroup& gr = groups[gi];
        if (gr.ranges.empty()) continue;
        if (unit_ms) PC_CUDA(cudaEventRecord(gev[2 * gi], s));
        PC_TRY(run_group(pg, gr, d_total, &launches, d_cost, d_tri, d_ecnt));
        if (unit_ms) PC_CUDA(cudaEventRecord(gev[2 * gi + 1], s));
    }
    PC_CUDA(cudaEventRecord(pg->ev1, s));
    unsigned long long h = 0;
    PC_CUDA(cudaMemcpyAsync(&h, d_total, 8, cudaMemcpyDeviceToHost, s));
    std::vector<unsigned long long> cyc(unit_ms ? U : 0);
    if (unit_ms && U) PC_CUDA(cudaMemcpyAsync(cyc.data(), d_cost, U * 8, cudaMemcpyDeviceToHost, s));
    const pc_status st = sync(pg);
    if (st != PC_OK) {
        drop_events();
        return st;
    }
    *count = h;
    if (unit_ms) {
        unit_ms->assign(U, 0.0);
        std::vector<double> gsum(groups.size(), 0.0), gms(groups.size(), 0.0);
        for (size_t u = 0; u < U; ++u)
            if (group_of[u] >= 0) gsum[group_of[u]] += (double)cyc[u];
        for (size_t gi = 0; gi < groups.size(); ++gi) {
            if (groups[gi].ranges.empty()) continue;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, gev[2 * gi], gev[2 * gi + 1]);
            gms[gi] = ms;
        }
        for (size_t u = 0; u < U; ++u) {
            const int gi = group_of[u];
            if (gi >= 0 && gsum[gi] > 0) (*unit_ms)[u] = gms[gi] * (double)cyc[u] / gsum[gi];
        }
        drop_events();
    }
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
        if (variant == PC_VARIANT_MATRIX && !pg->contiguous)
            return fail(PC_ERR_UNSUPPORTED, "forced matrix variant: the partitions are not contiguous id ranges");
        for (size_t u = 0; u < U; ++u) {
            const float* f = &feat[u * kNumFeatures];
            if (f[1] <= 0 || f[2] <= 0) continue;
            if (!variant_feasible(variant, f))
                return fail(PC_ERR_UNSUPPORTED, variant == PC_VARIANT_MATRIX
                                                    ? "forced matrix variant: a pivot id is 2^16 or above, or a unit's rows exceed 100 MB"
                                                    : "forced bitmap variant: a pivot id exceeds the shared-memory "
                                                      "bitmap capacity");
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
    HeuristicParams hp = heuristic_params();
    // the matrix form needs units that are id ranges
    if (!pg->contiguous) hp.matrix_scan = INFINITY;
    if (learned) PC_TRY(selector_choose_batch(feat, U, assign));
    for (size_t u = 0; u < U; ++u) {
        const float* f = &feat[u * kNumFeatures];
        if (f[1] <= 0 || f[2] <= 0) { (*assign)[u] = -1; continue; }
        int v = learned ? (*assign)[u] : heuristic_choice(f, hp);
        if (v < 0 || !variant_feasible(v, f) || (v == PC_VARIANT_MATRIX && !pg->contiguous))
            v = heuristic_choice(f, hp);
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

// Per-vertex triangle counts (each triangle adds 1 to each of its three
// vertices) into d_tri (n zeroed counters, outside the scratch arena) under
// the plan of `variant`; the matrix form has no per-vertex mode, so its units
// run with the 32-lane bitmap kernel.  Returns the triangle count.
pc_status tc_vertex_triangles(pc_pgraph* pg, int32_t variant, unsigned long long* d_tri, uint64_t* count) {
    PC_TRY(tc_ensure_features(pg));
    const size_t U = pg->unit_lo.size();
    *count = 0;
    if (U == 0 || pg->g->m == 0) return PC_OK;
    std::vector<int8_t> assign;
    int sel = 0;
    PC_TRY(tc_assign(pg, variant, pg->part_features, U, &assign, &sel));
    for (size_t u = 0; u < U; ++u) {
        if (assign[u] != PC_VARIANT_MATRIX) continue;
        const float* f = &pg->part_features[u * kNumFeatures];
        assign[u] = (int8_t)(bitmap_feasible(f) ? PC_VARIANT_BITMAP_WARP : PC_VARIANT_HASH_WARP);
    }
    return tc_execute(pg, assign, count, nullptr, nullptr, d_tri);
}

// Per-edge triangle counts at the oriented slots (the slot of edge {x, y},
// y < x, is the position of y in row x) into d_ecnt (m zeroed counters,
// outside the scratch arena), under the plan of `variant`; matrix units run
// with the 32-lane bitmap kernel.  Returns the triangle count.
pc_status tc_edge_triangles(pc_pgraph* pg, int32_t variant, uint32_t* d_ecnt, uint64_t* count) {
    PC_TRY(tc_ensure_features(pg));
    const size_t U = pg->unit_lo.size();
    *count = 0;
    if (U == 0 || pg->g->m == 0) return PC_OK;
    std::vector<int8_t> assign;
    int sel = 0;
    PC_TRY(tc_assign(pg, variant, pg->part_features, U, &assign, &sel));
    for (size_t u = 0; u < U; ++u) {
        if (assign[u] != PC_VARIANT_MATRIX) continue;
        const float* f = &pg->part_features[u * kNumFeatures];
        assign[u] = (int8_t)(bitmap_feasible(f) ? PC_VARIANT_BITMAP_WARP : PC_VARIANT_HASH_WARP);
    }
    return tc_execute(pg, assign, count, nullptr, nullptr, nullptr, d_ecnt);
}

// Runs one variant on every unit it can take (all units with work; bitmap
// variants only where the ids fit) in one profiled call; returns the per-unit
// cost inside that full run, -1 where the variant cannot run, and the count
// over the units it ran.
pc_status tc_profile_variant(pc_pgraph* pg, int variant, std::vector<double>* unit_ms, uint64_t* count) {
    PC_TRY(tc_ensure_features(pg));
    const size_t U = pg->unit_lo.size();
    std::vector<int8_t> assign(U, -1);
    const bool ok = variant != PC_VARIANT_MATRIX || pg->contiguous;
    for (size_t u = 0; u < U; ++u) {
        const float* f = &pg->part_features[u * kNumFeatures];
        if (ok && f[1] > 0 && f[2] > 0 && variant_feasible(variant, f)) assign[u] = (int8_t)variant;
    }
    PC_TRY(tc_execute(pg, assign, count, nullptr, unit_ms));
    for (size_t u = 0; u < U; ++u)
        if (assign[u] < 0) (*unit_ms)[u] = -1.0;
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
