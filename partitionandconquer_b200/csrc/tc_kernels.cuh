// Triangle-counting intersection kernels (sm_100a).
//
// Work decomposition ("pivot" form).  Orient every undirected edge from the
// larger id to the smaller id; with degree-descending ids this is the degree
// orientation.  Let N+(x) = N(x) & [0, x) -- the prefix of x's sorted row, of
// length dplus[x] -- and N-(x) the suffix (ids > x).  A triangle a < b < c is
// found exactly once, at pivot b and in-neighbour c in N-(b), as the element
// a of N(c) & [0, b) that is also in N+(b).  Hence
//     T = sum_b sum_{c in N-(b)} |N(c) & [0,b) & N+(b)|,
// the same number as the reference's sum over partitions of
// cnt_common_neis_less_than_merge(u, v, v, i) (src/Graph.cpp:1346-1362): both
// count every triangle once.  Every kernel processes all in-edges of a set
// of pivots, so kernels can be mixed per partition and the total stays exact.
//
// Work items are (pivot, run of in-neighbours) triples taken from a global
// counter, so hub pivots with 10^5 in-neighbours are spread over many CTAs.
//
// Pivot sets in shared memory:
//  * bitmap (CTA-wide): bit a set for a in N+(b), needs b <= capacity;
//  * split (CTA-wide): a bitmap of the ids below 2^16 and a hash of the rest
//    (SplitSet), for pivots past 2^16 in the count and per-vertex modes;
//  * hash (warp-private): open addressing, <= 256 keys in 512 slots;
//  * none: threshold merge (the reference's primitive) or binary search.
#pragma once
#include <stdint.h>

#include <type_traits>

#include "pc_internal.cuh"

namespace pc {
namespace tc {

constexpr int kTile = 16384;        // pivots per planning tile
constexpr int kChunkWarp = 256;     // in-neighbours per warp work item
constexpr int kCtaThreads = 512;    // threads per CTA of the bitmap kernels
constexpr int kHashSlots = 512;     // slots per warp-private hash table
constexpr int kHashCap = 256;       // max pivot set size for the hash kernel
constexpr int kWarpCtaWarps = 8;    // warps per CTA of the warp kernels
constexpr int kEcRankCap = 512;     // per-edge mode: pivot sets up to this size count by rank in shared memory
constexpr int kHubHist = 8192;      // per-vertex counting: ids below this count in shared memory

enum WarpMode { kModeHash = 0, kModeMerge = 1, kModeGallop = 2 };

struct Item {
    int32_t pos;  // plist position of the pivot
    int32_t j0;   // in-neighbours [j0, j1) of the pivot (indices into N-(b))
    int32_t j1;
};

__device__ __forceinline__ int32_t pivot_at(const int32_t* __restrict__ plist, int64_t p) {
    return plist ? plist[p] : (int32_t)p;
}

__device__ __forceinline__ uint32_t hash_slot(int32_t a) { return ((uint32_t)a * 0x9E3779B1u) >> (32 - 9); }

// Pivot sets the bitmap kernels test prefix ids against.
//
// BitmapSet: bit a of a shared-memory bitmap for every a in N+(b).
//
// SplitSet: ids below kSplitLo in a bitmap of kSplitLo bits (8 KB), ids at or
// above it in a 512-slot open-addressing hash.  The set's size no longer
// grows with the pivot's id, so units of pivots up to 2^20 keep 8 sets per
// CTA.  A pivot with more than kHashCap ids at or above kSplitLo does not fill
// the hash; its high ids are then found by binary search in N+(b) itself
// (`ovf`), so the test stays exact for every pivot.
constexpr int32_t kSplitLo = 1 << 16;
constexpr uint32_t kSplitWords = (uint32_t)kSplitLo / 32;

struct BitmapSet {
    const uint32_t* bm;
    __device__ __forceinline__ uint32_t test(int32_t a) const { return (bm[a >> 5] >> (a & 31)) & 1u; }
};

struct SplitSet {
    const uint32_t* bm;
    const int32_t* ht;             // kHashSlots slots, -1 = empty
    const int32_t* __restrict__ nb;  // N+(b) in the CSR (overflow path)
    uint32_t dp;
    bool ovf;
    __device__ __forceinline__ uint32_t test(int32_t a) const {
        if (a < kSplitLo) return (bm[a >> 5] >> (a & 31)) & 1u;
        if (ovf) {
            uint32_t lo = 0, hi = dp;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (__ldg(nb + mid) < a) lo = mid + 1; else hi = mid;
            }
            return (lo < dp && __ldg(nb + lo) == a) ? 1u : 0u;
        }
        uint32_t s = hash_slot(a);
        for (int32_t key; (key = ht[s]) != -1; s = (s + 1) & (kHashSlots - 1))
            if (key == a) return 1u;
        return 0u;
    }
};

// Named barrier over `nthreads` threads of one warp group (ids 1..15; id 0
// is __syncthreads).
__device__ __forceinline__ void group_barrier(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Per-vertex triangle counts (kVC): every triangle found adds 1 to its
// lowest vertex a; ids below kHubHist go to a shared-memory histogram
// (almost every hit is a hub), the rest to the global counts.
__device__ __forceinline__ void count_vertex(int32_t a, unsigned long long* __restrict__ tri, uint32_t* hist) {
    if (a < kHubHist) atomicAdd(&hist[a], 1u);
    else atomicAdd(&tri[a], 1ull);
}

// Position of a in the pivot set: bits of the bitmap below a, from the
// superblock prefix sb (one count per 8 words) and at most 8 word popcounts.
__device__ __forceinline__ uint32_t rank_in_set(const uint32_t* __restrict__ bm, const uint32_t* __restrict__ sb,
                                                int32_t a) {
    const uint32_t w = (uint32_t)a >> 5;
    uint32_t r = sb[w >> 3];
    for (uint32_t x = w & ~7u; x < w; ++x) r += __popc(bm[x]);
    return r + __popc(bm[w] & ((1u << (a & 31)) - 1u));
}

// Pipelined group-of-G prefix scan (the 32-lane groups use it): the load of
// the next G ids is issued before the current ones are tested, so two loads
// per lane are in flight.  Stops at the first id >= b and never reads past
// lim = dplus[c].
// Modes of the pivot-form kernels: count only; kVC per-vertex triangle
// counts (LCC); kEC per-edge counts at the oriented slots (Jaccard): every
// triangle a < b < c adds 1 to the slot of a in row c (its scan index), to
// the slot of a in row b (its rank in the pivot set) and, once per pair,
// its hits to the slot of b in row c (where the scan stops).
template <int G, bool kVC = false, bool kEC = false, class Set = BitmapSet>
__device__ __forceinline__ uint32_t scan_prefix_pipelined(const int32_t* __restrict__ row, uint32_t lim, int32_t b,
                                                          int gl, unsigned gmask, const Set& S,
                                                          unsigned long long* __restrict__ tri = nullptr,
                                                          uint32_t* hist = nullptr,
                                                          uint32_t* __restrict__ ec_c = nullptr,
                                                          uint32_t* __restrict__ ec_b = nullptr,
                                                          const uint32_t* __restrict__ sb = nullptr) {
    uint32_t hits = 0;
    uint32_t i = gl;
    int32_t kb = -1;  // kEC: index of b in the row, seen by one lane of the group
    int32_t a = i < lim ? __ldg(row + i) : 0x7fffffff;
    for (;;) {
        const uint32_t inext = i + G;
        const int32_t an = inext < lim ? __ldg(row + inext) : 0x7fffffff;
        if (a < b) {
            const uint32_t bit = S.test(a);
            hits += bit;
            if (kVC && bit) count_vertex(a, tri, hist);
            if (kEC && bit) {
                atomicAdd(&ec_c[i], 1u);
                atomicAdd(&ec_b[rank_in_set(S.bm, sb, a)], 1u);
            }
        } else if (kEC && a == b) {
            kb = (int32_t)i;
        }
        int32_t last;
        if constexpr (G == 1) last = a;
        else last = __shfl_sync(gmask, a, G - 1, G);
        if (last >= b) break;
        a = an;
        i = inext;
    }
    if (kEC) {
        const uint32_t total = G == 1 ? hits : __reduce_add_sync(gmask, hits);
        if (kb >= 0 && total) atomicAdd(&ec_c[kb], total);
    }
    return hits;
}

// The same scan with 16-byte loads, for groups of G < 32 lanes: each lane
// takes 4 consecutive ids per step, so a group of 8 reads a whole 128-byte
// line per dependent round instead of 32 bytes.  The row is read from the
// 16-byte boundary at or below its start (positions before 0 are masked);
// a load may run up to 3 ids past lim, which the adjacency array's padding
// (64 ids after the last row) keeps in bounds.
template <int G, bool kVC = false, bool kEC = false, class Set = BitmapSet>
__device__ __forceinline__ uint32_t scan_prefix_vec4(const int32_t* __restrict__ row, uint32_t lim, int32_t b, int gl,
                                                     unsigned gmask, const Set& S,
                                                     unsigned long long* __restrict__ tri = nullptr,
                                                     uint32_t* hist = nullptr, uint32_t* __restrict__ ec_c = nullptr,
                                                     uint32_t* __restrict__ ec_b = nullptr,
                                                     const uint32_t* __restrict__ sb = nullptr) {
    constexpr uint32_t kSpan = 4 * G;  // ids per group step
    const uint32_t mis = (uint32_t)(reinterpret_cast<uintptr_t>(row) >> 2) & 3u;
    const int4* q = reinterpret_cast<const int4*>(row - mis);
    const uint32_t total = lim + mis;  // ids from q[0] to the end of the bound
    const int4 none = make_int4(0x7fffffff, 0x7fffffff, 0x7fffffff, 0x7fffffff);
    uint32_t hits = 0;
    int32_t kb = -1;  // kEC: index of b in the row, seen by one lane of the group
    uint32_t c0 = 0;
    int4 v = 4u * gl < total ? __ldg(q + gl) : none;
    for (;;) {
        const uint32_t c1 = c0 + kSpan;
        const int4 vn = c1 + 4u * gl < total ? __ldg(q + c1 / 4 + gl) : none;
        const int32_t e[4] = {v.x, v.y, v.z, v.w};
        bool stop = false;
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int64_t pos = (int64_t)(c0 + 4u * gl + t) - (int64_t)mis;  // index in row
            if (pos < 0 || pos >= (int64_t)lim) continue;
            const int32_t a = e[t];
            if (a < b) {
                const uint32_t bit = S.test(a);
                hits += bit;
                if (kVC && bit) count_vertex(a, tri, hist);
                if (kEC && bit) {
                    atomicAdd(&ec_c[pos], 1u);
                    atomicAdd(&ec_b[rank_in_set(S.bm, sb, a)], 1u);
                }
            } else {
                stop = true;
                if (kEC && a == b) kb = (int32_t)pos;
            }
        }
        bool any_stop;
        if constexpr (G == 1) any_stop = stop;
        else any_stop = __any_sync(gmask, stop);
        if (any_stop || c1 >= total) break;
        v = vn;
        c0 = c1;
    }
    if (kEC) {
        const uint32_t sum = G == 1 ? hits : __reduce_add_sync(gmask, hits);
        if (kb >= 0 && sum) atomicAdd(&ec_c[kb], sum);
    }
    return hits;
}

// The prefix scan a group of G lanes runs: 16-byte loads below 32 lanes.
template <int G, bool kVC = false, bool kEC = false, class Set = BitmapSet>
__device__ __forceinline__ uint32_t scan_group_prefix(const int32_t* __restrict__ row, uint32_t lim, int32_t b, int gl,
                                                      unsigned gmask, const Set& S,
                                                      unsigned long long* __restrict__ tri = nullptr,
                                                      uint32_t* hist = nullptr, uint32_t* __restrict__ ec_c = nullptr,
                                                      uint32_t* __restrict__ ec_b = nullptr,
                                                      const uint32_t* __restrict__ sb = nullptr) {
    if constexpr (G < 32) return scan_prefix_vec4<G, kVC, kEC>(row, lim, b, gl, gmask, S, tri, hist, ec_c, ec_b, sb);
    else return scan_prefix_pipelined<G, kVC, kEC>(row, lim, b, gl, gmask, S, tri, hist, ec_c, ec_b, sb);
}

// Bitmap kernel: a CTA of kCtaThreads threads holds 16/K pivot sets in
// shared memory, one per group of K warps; each group takes its own work
// items (pivot, a run of its in-neighbours), so a group synchronises only
// with itself (a named barrier, or nothing when K == 1).  In-neighbour metadata
// (id, row offset, prefix length) is fetched 32 at a time with one coalesced
// load and 32 independent gathers, then handed to groups of G lanes by
// shuffles; each group scans one prefix with scan_group_prefix.
// With kSplit the sets are SplitSets: bm_words = kSplitWords bitmap words,
// then kHashSlots hash slots, whatever the pivots' ids (count and per-vertex
// modes; the per-edge mode needs ranks in a plain bitmap).
template <int K, int G, bool kVC = false, bool kEC = false, bool kSplit = false>
__global__ void __launch_bounds__(kCtaThreads) k_tc_bitmap(const uint64_t* __restrict__ off,
                                                           const int32_t* __restrict__ adj,
                                                           const uint32_t* __restrict__ dplus,
                                                           const int32_t* __restrict__ plist,
                                                           const Item* __restrict__ items,
                                                           const uint32_t* __restrict__ nitems_p,
                                                           uint32_t* __restrict__ next_item,
                                                           unsigned long long* __restrict__ total,
                                                           uint32_t bm_words,
                                                           unsigned long long* __restrict__ unit_cost,
                                                           const int32_t* __restrict__ unit_of,
                                                           unsigned long long* __restrict__ tri = nullptr,
                                                           uint32_t* __restrict__ ecnt = nullptr) {
    static_assert(!(kSplit && kEC), "per-edge counts need the plain bitmap's ranks");
    extern __shared__ uint32_t smem[];
    __shared__ uint32_t s_item[16];
    __shared__ uint32_t s_hic[16];  // kSplit: ids >= kSplitLo offered to the set's hash this item
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int set = warp / K, wi = warp % K;
    const int nsets = (kCtaThreads / 32) / K;
    const int set_threads = K * 32, tis = wi * 32 + lane;
    const uint32_t set_words = bm_words + (kSplit ? (uint32_t)kHashSlots : 0u);
    uint32_t* bm = smem + (size_t)set * set_words;
    int32_t* ht = reinterpret_cast<int32_t*>(bm + bm_words);  // kSplit: the set's hash slots
    uint32_t* hist = smem + (size_t)nsets * set_words;  // kVC: kHubHist counters after the sets
    // kEC: per set, the rank of the first pivot-set entry of every touched
    // 256-id superblock (only those are ever read)
    const uint32_t nsb = (bm_words + 7) / 8;
    uint32_t* sb = smem + (size_t)nsets * bm_words + (size_t)set * nsb;
    // kEC: per set, hits by rank in the pivot set (sets up to kEcRankCap),
    // flushed to the row's slots once per item
    uint32_t* ecs = smem + (size_t)nsets * (bm_words + nsb) + (size_t)set * kEcRankCap;
    const uint32_t zero_words = (uint32_t)nsets * set_words + (kVC ? (uint32_t)kHubHist : 0u);
    for (uint32_t i = tid; i < zero_words; i += blockDim.x)
        smem[i] = (kSplit && i < (uint32_t)nsets * set_words && i % set_words >= bm_words) ? 0xffffffffu : 0u;
    if (kEC)
        for (uint32_t i = tid; i < (uint32_t)nsets * kEcRankCap; i += blockDim.x)
            smem[(size_t)nsets * (bm_words + nsb) + i] = 0;
    if (tid < 16) s_hic[tid] = 0;
    __syncthreads();
    auto set_sync = [&]() {
        if constexpr (K == 1) __syncwarp();
        else group_barrier(1 + set, set_threads);
    };
    const uint32_t nitems = *nitems_p;
    constexpr int NG = 32 / G;  // in-neighbours handled at once per warp
    const int gidx = lane / G, gl = lane % G;
    const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (lane & ~(G - 1)));
    unsigned long long cnt = 0;
    for (;;) {
        if (tis == 0) s_item[set] = atomicAdd(next_item, 1u);
        set_sync();
        const uint32_t it = s_item[set];
        if (it >= nitems) break;
        const long long t0 = unit_cost ? clock64() : 0;
        const Item I = items[it];
        const int32_t b = pivot_at(plist, I.pos);
        const uint64_t rb = off[b], re = off[b + 1];
        const uint32_t dp = dplus[b];
        for (uint32_t k = tis; k < dp; k += set_threads) {
            const int32_t a = adj[rb + k];
            if (!kSplit || a < kSplitLo) {
                atomicOr(&bm[a >> 5], 1u << (a & 31));
            } else if (atomicAdd(&s_hic[set], 1u) < (uint32_t)kHashCap) {
                // at most kHashCap keys in kHashSlots slots: a free slot exists
                uint32_t hs = hash_slot(a);
                while (atomicCAS(&ht[hs], -1, a) != -1) hs = (hs + 1) & (kHashSlots - 1);
            }
            if (kEC && (k == 0 || (adj[rb + k - 1] >> 8) != (a >> 8))) sb[a >> 8] = k;
        }
        set_sync();
        const uint32_t hic = kSplit ? s_hic[set] : 0u;
        std::conditional_t<kSplit, SplitSet, BitmapSet> S;
        if constexpr (kSplit) S = SplitSet{bm, ht, adj + rb, dp, hic > (uint32_t)kHashCap};
        else S = BitmapSet{bm};
        const uint64_t in0 = rb + dp + (uint64_t)I.j0;
        const uint64_t in1 = min(rb + dp + (uint64_t)I.j1, re);
        unsigned long long hb = 0;  // kVC: this item's triangles at pivot b
        for (uint64_t base = in0 + (uint64_t)wi * 32; base < in1; base += (uint64_t)set_threads) {
            const uint64_t e = base + lane;
            const bool ok = e < in1;
            const int32_t c = ok ? adj[e] : 0;
            const uint64_t rc = ok ? off[c] : 0;
            const uint32_t lim = ok ? dplus[c] : 0;
            const uint64_t left = in1 - base;
            const int nb = left < 32 ? (int)left : 32;
            for (int j0 = 0; j0 < 32; j0 += NG) {
                if (j0 >= nb) break;
                const int j = j0 + gidx;
                const int src = j < nb ? j : 0;
                const uint64_t rcj = __shfl_sync(0xffffffffu, rc, src);
                uint32_t limj = __shfl_sync(0xffffffffu, lim, src);
                if (j >= nb) limj = 0;
                if (kEC) {
                    if (limj) cnt += scan_group_prefix<G, false, true>(adj + rcj, limj, b, gl, gmask, S, nullptr,
                                                                           nullptr, ecnt + rcj,
                                                                           dp <= kEcRankCap ? ecs : ecnt + rb, sb);
                } else if (kVC) {
                    const int32_t cj = __shfl_sync(0xffffffffu, c, src);
                    if (limj) {
                        const uint32_t h = scan_group_prefix<G, true>(adj + rcj, limj, b, gl, gmask, S, tri, hist);
                        cnt += h;
                        hb += h;
                        if (h) atomicAdd(&tri[cj], (unsigned long long)h);
                    }
                } else if (limj) {
                    cnt += scan_group_prefix<G>(adj + rcj, limj, b, gl, gmask, S);
                }
            }
        }
        if (kVC) {
            for (int o = 16; o; o >>= 1) hb += __shfl_xor_sync(0xffffffffu, hb, o);
            if (lane == 0 && hb) atomicAdd(&tri[b], hb);
        }
        set_sync();
        for (uint32_t k = tis; k < dp; k += set_threads) {
            const int32_t a = adj[rb + k];
            if (!kSplit || a < kSplitLo) bm[a >> 5] = 0;
            if (kEC && dp <= kEcRankCap) {
                const uint32_t h = ecs[k];
                if (h) {
                    atomicAdd(&ecnt[rb + k], h);
                    ecs[k] = 0;
                }
            }
        }
        if (kSplit && hic) {
            for (uint32_t x = tis; x < (uint32_t)kHashSlots; x += set_threads) ht[x] = -1;
            if (tis == 0) s_hic[set] = 0;  // every lane read it before the scan barrier
        }
        set_sync();
        // profiling runs: the set's warp-cycles on this item, charged to its unit
        if (unit_cost && tis == 0) atomicAdd(&unit_cost[unit_of[b]], (unsigned long long)(clock64() - t0) * K);
    }
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0 && cnt) atomicAdd(total, cnt);
    if (kVC) {
        __syncthreads();
        for (uint32_t i = tid; i < (uint32_t)kHubHist; i += blockDim.x)
            if (hist[i]) atomicAdd(&tri[i], (unsigned long long)hist[i]);
    }
}

// |x & y & [0, thr)| for sorted x, y: Partitioned_Graph::
// cnt_common_neis_less_than_merge (src/Graph.cpp:1132-1153), without its
// one-past-the-end reads.
__device__ __forceinline__ uint32_t merge_below(const int32_t* __restrict__ x, uint32_t nx,
                                                const int32_t* __restrict__ y, uint32_t ny, int32_t thr) {
    uint32_t i = 0, j = 0, c = 0;
    while (i < nx && j < ny) {
        const int32_t a = x[i], bb = y[j];
        if (a >= thr || bb >= thr) break;
        if (a < bb) ++i;
        else if (a > bb) ++j;
        else { ++c; ++i; ++j; }
    }
    return c;
}

// Each id of N(c) & [0, thr) looked up in N+(b) by binary search: the
// lower_bound probing of Partitioned_Graph::cnt_common_neis_galloping
// (src/Graph.cpp:1071-1085).
__device__ __forceinline__ uint32_t gallop_below(const int32_t* __restrict__ x, uint32_t nx,
                                                 const int32_t* __restrict__ y, uint32_t ny, int32_t thr) {
    uint32_t c = 0;
    for (uint32_t i = 0; i < nx; ++i) {
        const int32_t a = x[i];
        if (a >= thr) break;
        uint32_t lo = 0, hi = ny;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (y[mid] < a) lo = mid + 1; else hi = mid;
        }
        c += (lo < ny && y[lo] == a) ? 1u : 0u;
    }
    return c;
}

// merge_below / gallop_below with per-vertex counting of every match (kVC).
template <bool kVC>
__device__ __forceinline__ uint32_t merge_below_vc(const int32_t* __restrict__ x, uint32_t nx,
                                                   const int32_t* __restrict__ y, uint32_t ny, int32_t thr,
                                                   unsigned long long* __restrict__ tri, uint32_t* hist) {
    uint32_t i = 0, j = 0, c = 0;
    while (i < nx && j < ny) {
        const int32_t a = x[i], bb = y[j];
        if (a >= thr || bb >= thr) break;
        if (a < bb) ++i;
        else if (a > bb) ++j;
        else {
            ++c;
            if (kVC) count_vertex(a, tri, hist);
            ++i;
            ++j;
        }
    }
    return c;
}

template <bool kVC>
__device__ __forceinline__ uint32_t gallop_below_vc(const int32_t* __restrict__ x, uint32_t nx,
                                                    const int32_t* __restrict__ y, uint32_t ny, int32_t thr,
                                                    unsigned long long* __restrict__ tri, uint32_t* hist) {
    uint32_t c = 0;
    for (uint32_t i = 0; i < nx; ++i) {
        const int32_t a = x[i];
        if (a >= thr) break;
        uint32_t lo = 0, hi = ny;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (y[mid] < a) lo = mid + 1; else hi = mid;
        }
        if (lo < ny && y[lo] == a) {
            ++c;
            if (kVC) count_vertex(a, tri, hist);
        }
    }
    return c;
}

// Per-edge forms (kEC): matches add 1 to the slots of a in row c (x) and in
// the pivot set (y); the pair's total goes to the slot of b = thr in x.
__device__ __forceinline__ uint32_t merge_below_ec(const int32_t* __restrict__ x, uint32_t nx,
                                                   const int32_t* __restrict__ y, uint32_t ny, int32_t thr,
                                                   uint32_t* __restrict__ ec_x, uint32_t* __restrict__ ec_y) {
    uint32_t i = 0, j = 0, c = 0;
    while (i < nx && j < ny) {
        const int32_t a = x[i], bb = y[j];
        if (a >= thr || bb >= thr) break;
        if (a < bb) ++i;
        else if (a > bb) ++j;
        else {
            ++c;
            atomicAdd(&ec_x[i], 1u);
            atomicAdd(&ec_y[j], 1u);
            ++i;
            ++j;
        }
    }
    while (i < nx && x[i] < thr) ++i;
    if (c && i < nx) atomicAdd(&ec_x[i], c);  // x[i] == thr: thr is in x
    return c;
}

__device__ __forceinline__ uint32_t gallop_below_ec(const int32_t* __restrict__ x, uint32_t nx,
                                                    const int32_t* __restrict__ y, uint32_t ny, int32_t thr,
                                                    uint32_t* __restrict__ ec_x, uint32_t* __restrict__ ec_y) {
    uint32_t c = 0, i = 0;
    for (; i < nx; ++i) {
        const int32_t a = x[i];
        if (a >= thr) break;
        uint32_t lo = 0, hi = ny;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (y[mid] < a) lo = mid + 1; else hi = mid;
        }
        if (lo < ny && y[lo] == a) {
            ++c;
            atomicAdd(&ec_x[i], 1u);
            atomicAdd(&ec_y[lo], 1u);
        }
    }
    if (c && i < nx) atomicAdd(&ec_x[i], c);
    return c;
}

// Warp kernels: one item (pivot, <= kChunkWarp in-neighbours) per warp, one
// lane per in-neighbour.
template <int MODE, bool kVC = false, bool kEC = false>
__global__ void __launch_bounds__(kWarpCtaWarps * 32) k_tc_warp(const uint64_t* __restrict__ off,
                                                                const int32_t* __restrict__ adj,
                                                                const uint32_t* __restrict__ dplus,
                                                                const int32_t* __restrict__ plist,
                                                                const Item* __restrict__ items,
                                                                const uint32_t* __restrict__ nitems_p,
                                                                uint32_t* __restrict__ next_item,
                                                                unsigned long long* __restrict__ total,
                                                                unsigned long long* __restrict__ unit_cost,
                                                                const int32_t* __restrict__ unit_of,
                                                                unsigned long long* __restrict__ tri = nullptr,
                                                                uint32_t* __restrict__ ecnt = nullptr) {
    __shared__ int32_t table[MODE == kModeHash ? kWarpCtaWarps : 1][MODE == kModeHash ? kHashSlots : 1];
    __shared__ int32_t tpos[MODE == kModeHash && kEC ? kWarpCtaWarps : 1][MODE == kModeHash && kEC ? kHashSlots : 1];
    // kEC: per warp, the hits of the pivot set's entries by rank, flushed to
    // their slots once per item instead of one global atomic per triangle
    __shared__ uint32_t rcnt[MODE == kModeHash && kEC ? kWarpCtaWarps : 1][MODE == kModeHash && kEC ? kHashCap : 1];
    __shared__ uint32_t hist[kVC ? kHubHist : 1];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t* T = table[MODE == kModeHash ? w : 0];
    int32_t* TP = tpos[MODE == kModeHash && kEC ? w : 0];  // kEC: position of each key in N+(b)
    uint32_t* RC = rcnt[MODE == kModeHash && kEC ? w : 0];
    if (kVC) {
        for (int i = threadIdx.x; i < kHubHist; i += blockDim.x) hist[i] = 0;
        __syncthreads();
    }
    if (MODE == kModeHash) {
        for (int s = lane; s < kHashSlots; s += 32) T[s] = -1;
        if (kEC)
            for (int s = lane; s < kHashCap; s += 32) RC[s] = 0;
        __syncwarp();
    }
    const uint32_t nitems = *nitems_p;
    unsigned long long cnt = 0;
    for (;;) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(next_item, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= nitems) break;
        const long long t0 = unit_cost ? clock64() : 0;
        const unsigned long long cnt_item0 = cnt;
        const Item I = items[it];
        const int32_t b = pivot_at(plist, I.pos);
        const uint64_t rb = off[b], re = off[b + 1];
        const uint32_t dp = dplus[b];
        const uint64_t in0 = rb + dp + (uint64_t)I.j0;
        const uint64_t in1 = min(rb + dp + (uint64_t)I.j1, re);
        const int32_t* nb = adj + rb;
        if (MODE == kModeHash && dp <= (uint32_t)kHashCap) {
            for (uint32_t k = lane; k < dp; k += 32) {
                const int32_t a = nb[k];
                uint32_t s = hash_slot(a);
                while (atomicCAS(&T[s], -1, a) != -1) s = (s + 1) & (kHashSlots - 1);
                if (kEC) TP[s] = (int32_t)k;
            }
            __syncwarp();
            for (uint64_t e = in0 + lane; e < in1; e += 32) {
                const int32_t c = adj[e];
                const uint64_t rc = off[c];
                const int32_t* row = adj + rc;
                const uint32_t lim = dplus[c];
                // the lane's prefix scan, 4 ids per 16-byte load with the
                // next load in flight (read from the 16-byte boundary at or
                // below the row start; the padding after the last row keeps
                // the up to 3 ids past lim in bounds)
                uint32_t h = 0, i = lim;  // i: index of the first id >= b
                const uint32_t mis = (uint32_t)(reinterpret_cast<uintptr_t>(row) >> 2) & 3u;
                const int4* q = reinterpret_cast<const int4*>(row - mis);
                const uint32_t total = lim + mis;
                int4 v = total ? __ldg(q) : make_int4(0, 0, 0, 0);
                bool stop = false;
                // one id of the prefix at index pos (masked outside [0, lim))
                auto probe = [&](int32_t a, int64_t pos) {
                    if (stop || pos < 0 || pos >= (int64_t)lim) return;
                    if (a >= b) {
                        stop = true;
                        i = (uint32_t)pos;
                        return;
                    }
                    uint32_t s = hash_slot(a);
                    int32_t key;
                    while ((key = T[s]) != -1) {
                        if (key == a) {
                            ++h;
                            if (kVC) count_vertex(a, tri, hist);
                            if (kEC) {
                                atomicAdd(&ecnt[rc + pos], 1u);
                                atomicAdd(&RC[TP[s]], 1u);
                            }
                            break;
                        }
                        s = (s + 1) & (kHashSlots - 1);
                    }
                };
                for (uint32_t c0 = 0; c0 < total; c0 += 4) {
                    const int4 vn = c0 + 4 < total ? __ldg(q + c0 / 4 + 1) : v;
                    const int64_t p0 = (int64_t)c0 - (int64_t)mis;
                    probe(v.x, p0);
                    probe(v.y, p0 + 1);
                    probe(v.z, p0 + 2);
                    probe(v.w, p0 + 3);
                    if (stop) break;
                    v = vn;
                }
                cnt += h;
                if (kVC && h) atomicAdd(&tri[c], (unsigned long long)h);
                if (kEC && h && i < lim) atomicAdd(&ecnt[rc + i], h);  // row[i] == b
            }
            __syncwarp();
            for (int s = lane; s < kHashSlots; s += 32) T[s] = -1;
            if (kEC) {
                for (uint32_t k = lane; k < dp; k += 32) {
                    const uint32_t h = RC[k];
                    if (h) {
                        atomicAdd(&ecnt[rb + k], h);
                        RC[k] = 0;
                    }
                }
            }
            __syncwarp();
        } else if (MODE == kModeGallop) {
            for (uint64_t e = in0 + lane; e < in1; e += 32) {
                const int32_t c = adj[e];
                if (kEC) {
                    const uint64_t rc = off[c];
                    cnt += gallop_below_ec(adj + rc, dplus[c], nb, dp, b, ecnt + rc, ecnt + rb);
                    continue;
                }
                const uint32_t h = gallop_below_vc<kVC>(adj + off[c], dplus[c], nb, dp, b, tri, hist);
                cnt += h;
                if (kVC && h) atomicAdd(&tri[c], (unsigned long long)h);
            }
        } else {
            for (uint64_t e = in0 + lane; e < in1; e += 32) {
                const int32_t c = adj[e];
                if (kEC) {
                    const uint64_t rc = off[c];
                    cnt += merge_below_ec(adj + rc, dplus[c], nb, dp, b, ecnt + rc, ecnt + rb);
                    continue;
                }
                const uint32_t h = merge_below_vc<kVC>(adj + off[c], dplus[c], nb, dp, b, tri, hist);
                cnt += h;
                if (kVC && h) atomicAdd(&tri[c], (unsigned long long)h);
            }
        }
        if (unit_cost) {
            __syncwarp();
            if (lane == 0) atomicAdd(&unit_cost[unit_of[b]], (unsigned long long)(clock64() - t0));
        }
        if (kVC) {
            // this item's triangles at pivot b: the warp's hits since the item began
            unsigned long long hb = cnt - cnt_item0;
            for (int o = 16; o; o >>= 1) hb += __shfl_xor_sync(0xffffffffu, hb, o);
            if (lane == 0 && hb) atomicAdd(&tri[b], hb);
        }
    }
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0 && cnt) atomicAdd(total, cnt);
    if (kVC) {
        __syncthreads();
        for (int i = threadIdx.x; i < kHubHist; i += blockDim.x)
            if (hist[i]) atomicAdd(&tri[i], (unsigned long long)hist[i]);
    }
}


// ---- in-neighbour-major form for hub units (variant "matrix") ----------------
//
// For a unit of pivots b in the id range [lo, hi) (hi <= kMatrixMaxId), the
// pivot sets N+(b) are kept as bitmap rows H[b - lo] of hi bits in global
// memory: (hi - lo) * hi / 8 bytes, 32 MB for the first 16 K ids, which stay
// in L2.  The kernel then walks the in-neighbours c instead of the pivots:
// S_c = N(c) & [0, min(hi, c)) is read once, and for every pivot b in
// S_c & [lo, hi) at position j of S_c the count |S_c[0..j) & N+(b)| is taken
// either by j bit probes into H[b] or by ceil(b/32) word-wise ANDs of H[b]
// with a shared-memory bitmap of S_c and popcounts, whichever is cheaper.
// Every (pivot, in-neighbour) pair of the unit is one pair (b, c) here, so the
// count equals the pivot form's; what changes is that N(c) comes from DRAM
// once per c instead of once per pivot.
constexpr int kMatrixMaxId = 1 << 16;      // hi bound: rows of <= 8 KB, H <= 512 MB
constexpr int kMatrixWarps = 8;            // warps per CTA
constexpr int kMatrixWordsMax = kMatrixMaxId / 32;

__device__ __forceinline__ uint32_t lower_bound_i32(const int32_t* __restrict__ p, uint32_t n, int32_t x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (p[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

}  // namespace tc
}  // namespace pc
