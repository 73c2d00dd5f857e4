// Frontier algorithms: BFS, SSSP, PageRank, k-core, MIS, CDLP (sm_100a).
//
// All kernels work on the symmetric CSR in the internal id space; inputs and
// outputs are mapped to the caller's id space (identity unless the view was
// reordered).  Frontiers are compacted queues; appends are warp-aggregated
// (one atomic per warp and step).
#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include <cub/block/block_scan.cuh>

#include "grid_sync.cuh"
#include "pc_internal.cuh"
#include "synth_rng.h"

namespace pc {
namespace fr {

constexpr int kThreads = 256;
constexpr int32_t kInf = INT_MAX;
// bound on any grid-barrier wait of the persistent kernels (4 s)
constexpr uint64_t kBarrierLimitNs = 4000000000ull;
// k-core: ids below this have their degree decrements gathered per CTA
constexpr int kKcoreHubs = 4096;
constexpr uint32_t kLocalQ = 1024;       // k-core: per-CTA queue of vertices pushed in a step
constexpr uint32_t kLocalEdges = 16384;  // ... peeled by the CTA itself while their rows stay below this
static_assert(kKcoreHubs % kThreads == 0, "the flush loop needs a uniform trip count");

// Appends `val` for every lane with pred set; all 32 lanes of the warp must
// call it together.
__device__ __forceinline__ void warp_append(bool pred, int32_t val, int32_t* __restrict__ q,
                                            uint32_t* __restrict__ qn) {
    const unsigned m = __ballot_sync(0xffffffffu, pred);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(qn, (uint32_t)__popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (pred) q[base + __popc(m & ((1u << lane) - 1u))] = val;
}

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t x) {
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// ---- rows longer than kHeavyDeg ------------------------------------------------
// A warp-per-vertex loop serialises a hub's row on one warp (RMAT-22's largest
// row has 163K entries: 5100 rounds of dependent loads on one warp).  The
// frontier kernels set such vertices aside in a heavy list; heavy_rows() then
// spreads the rows of the list over every warp of the grid in chunks of
// kHeavyChunk entries, balanced by a block-local prefix of chunk counts.
constexpr uint32_t kHeavyDeg = 1024;
constexpr uint32_t kHeavyChunk = 256;
constexpr uint32_t kHeavyBatch = 2048;  // list entries per shared-memory prefix
static_assert(kHeavyBatch % kThreads == 0, "prefix items per thread");
// Pull kernels (PageRank, CDLP): rows of more than kPullHeavyDeg entries get a
// CTA; the others kPullLanes lanes, so a warp keeps 8 rows in flight (4 lanes
// measured 10 % faster than 8 for PageRank at RMAT-22, 16 lanes 16 % slower).
constexpr uint32_t kPullHeavyDeg = 256;
constexpr int kPullLanes = 4;
constexpr int kMisLanes = 8;  // MIS under id priorities: lanes per vertex

// Calls body(u, j, valid) for the entries j of every row of hq[0..hn); the 32
// lanes of a warp call it together (valid is false past a row's end), so the
// body may use warp collectives.  All threads of every CTA must call it.
template <class Body>
__device__ __forceinline__ void heavy_rows(const uint64_t* __restrict__ off, const int32_t* hq, uint32_t hn,
                                           Body&& body) {
    using Scan = cub::BlockScan<uint32_t, kThreads>;
    __shared__ typename Scan::TempStorage scan_tmp;
    __shared__ uint32_t s_pref[kHeavyBatch + 1];
    constexpr int kPer = kHeavyBatch / kThreads;
    const int lane = threadIdx.x & 31;
    const uint64_t wpb = blockDim.x >> 5;
    const uint64_t gw = blockIdx.x * wpb + (threadIdx.x >> 5), nw = (uint64_t)gridDim.x * wpb;
    for (uint32_t h0 = 0; h0 < hn; h0 += kHeavyBatch) {
        const uint32_t hb = min(kHeavyBatch, hn - h0);
        uint32_t cnt[kPer];
        for (int t = 0; t < kPer; ++t) {
            const uint32_t h = threadIdx.x * kPer + t;
            cnt[t] = 0;
            if (h < hb) {
                const int32_t u = __ldcg(hq + h0 + h);
                cnt[t] = (uint32_t)((off[u + 1] - off[u] + kHeavyChunk - 1) / kHeavyChunk);
            }
        }
        __syncthreads();  // the previous batch is done with s_pref and scan_tmp
        uint32_t total = 0;
        Scan(scan_tmp).ExclusiveSum(cnt, cnt, total);
        for (int t = 0; t < kPer; ++t) s_pref[threadIdx.x * kPer + t] = cnt[t];
        if (threadIdx.x == 0) s_pref[kHeavyBatch] = total;
        __syncthreads();
        for (uint64_t c = gw; c < total; c += nw) {
            uint32_t lo = 0, hi = hb - 1;  // last row whose chunks start at or before c
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1) >> 1;
                if (s_pref[mid] <= c) lo = mid; else hi = mid - 1;
            }
            const int32_t u = __ldcg(hq + h0 + lo);
            const uint64_t rb = off[u] + (c - s_pref[lo]) * (uint64_t)kHeavyChunk;
            const uint64_t re = min(rb + kHeavyChunk, off[u + 1]);
            for (uint64_t j0 = rb; j0 < re; j0 += 32) body(u, j0 + lane, j0 + lane < re);
        }
    }
}

// Rows of more than thr entries (the pull kernels give each a whole CTA).
__global__ void k_heavy_list(const uint64_t* __restrict__ off, uint64_t n, uint32_t thr, int32_t* __restrict__ hq,
                             uint32_t* __restrict__ hn) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t nr = (n + 31) & ~31ull;
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < nr; u += stride) {
        const bool heavy = u < n && off[u + 1] - off[u] > thr;
        warp_append(heavy, (int32_t)u, hq, hn);
    }
}

// ---- BFS -------------------------------------------------------------------

__global__ void k_iota(int32_t* a, uint64_t n) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) a[i] = (int32_t)i;
}

__global__ void k_fill_i32(int32_t* a, uint64_t n, int32_t v) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

// Top-down step: one warp per frontier vertex, lanes over its neighbours.
__global__ void k_bfs_top_down(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                               const int32_t* __restrict__ fq, uint32_t fn, int32_t* __restrict__ dist,
                               int32_t level, int32_t* __restrict__ nq, uint32_t* __restrict__ nn,
                               unsigned long long* __restrict__ next_edges, int32_t* __restrict__ hq,
                               uint32_t* __restrict__ hn) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    uint64_t edges = 0;
    for (uint64_t i = warp; i < fn; i += nwarps) {
        const int32_t u = fq[i];
        const uint64_t b = off[u], e = off[u + 1];
        if (e - b > kHeavyDeg) {  // expanded by k_bfs_top_down_heavy
            if (lane == 0) hq[atomicAdd(hn, 1u)] = u;
            continue;
        }
        for (uint64_t j0 = b; j0 < e; j0 += 32) {
            const uint64_t j = j0 + lane;
            bool won = false;
            int32_t v = 0;
            if (j < e) {
                v = adj[j];
                if (dist[v] == kInf) won = atomicCAS(&dist[v], kInf, level) == kInf;
            }
            if (won) edges += off[v + 1] - off[v];
            warp_append(won, v, nq, nn);
        }
    }
    edges = warp_sum_u64(edges);
    if (lane == 0 && edges) atomicAdd(next_edges, (unsigned long long)edges);
}

// The heavy frontier vertices of a top-down step, spread over the grid.
__global__ void k_bfs_top_down_heavy(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                                     const int32_t* __restrict__ hq, const uint32_t* __restrict__ hn,
                                     int32_t* __restrict__ dist, int32_t level, int32_t* __restrict__ nq,
                                     uint32_t* __restrict__ nn, unsigned long long* __restrict__ next_edges) {
    uint64_t edges = 0;
    heavy_rows(off, hq, *hn, [&](int32_t, uint64_t j, bool ok) {
        bool won = false;
        int32_t v = 0;
        if (ok) {
            v = adj[j];
            if (dist[v] == kInf) won = atomicCAS(&dist[v], kInf, level) == kInf;
        }
        if (won) edges += off[v + 1] - off[v];
        warp_append(won, v, nq, nn);
    });
    edges = warp_sum_u64(edges);
    if ((threadIdx.x & 31) == 0 && edges) atomicAdd(next_edges, (unsigned long long)edges);
}

// Bottom-up step: every unvisited vertex looks for a neighbour at level-1.
__global__ void k_bfs_bottom_up(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj, uint64_t n,
                                int32_t* __restrict__ dist, int32_t level, int32_t* __restrict__ nq,
                                uint32_t* __restrict__ nn, unsigned long long* __restrict__ next_edges) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t nr = (n + 31) & ~31ull;
    uint64_t edges = 0;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < nr; v += stride) {
        bool found = false;
        if (v < n && dist[v] == kInf) {
            const uint64_t b = off[v], e = off[v + 1];
            for (uint64_t j = b; j < e; ++j) {
                if (dist[adj[j]] == level - 1) { found = true; break; }
            }
            if (found) {
                dist[v] = level;
                edges += e - b;
            }
        }
        warp_append(found, (int32_t)v, nq, nn);
    }
    edges = warp_sum_u64(edges);
    if ((threadIdx.x & 31) == 0 && edges) atomicAdd(next_edges, (unsigned long long)edges);
}

__global__ void k_bfs_finish(const int32_t* __restrict__ dist, uint64_t n, int32_t* __restrict__ rank) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) rank[i] = dist[i] == 0 ? -1 : dist[i];
}

// ---- SSSP: frontier Bellman-Ford and delta-stepping --------------------------
//
// Both forms relax the rows of a frontier with atomicMin and queue every
// vertex whose distance falls; they differ in which improved vertices are
// relaxed next.  Bellman-Ford (kDelta = false) relaxes all of them in the
// next round.  Delta-stepping (kDelta = true; Meyer and Sanders, "Delta-
// stepping: a parallelizable shortest path algorithm", J. Algorithms 2003, in
// the near/far-pile form of Davidson, Baxter, Garland and Owens, IPDPS 2014)
// relaxes only vertices whose new distance is below the current bucket's
// upper bound `thr` ("near"); the others go to a far pile that is split when
// the bucket is exhausted.  Both are label-correcting: every improvement is
// queued, so both end at the exact shortest distances (integer weights >= 0).
struct SsspPush {
    int32_t thr;                 // delta-stepping: near bound (exclusive)
    int32_t* __restrict__ far;   // far pile and its length
    uint32_t* __restrict__ farn;
    int32_t* __restrict__ farflag;  // 1 while the vertex is in the far pile
};

template <bool kDelta>
__device__ __forceinline__ void sssp_relax_edge(int32_t du, int32_t v, int32_t wt, int32_t* __restrict__ dist,
                                                int32_t* __restrict__ flag, const SsspPush& P, bool* near,
                                                bool* far) {
    const int32_t nd = du + wt;
    if (nd < dist[v]) {
        const int32_t old = atomicMin(&dist[v], nd);
        if (nd < old) {
            if (!kDelta || nd < P.thr) *near = atomicExch(&flag[v], 1) == 0;
            else *far = atomicExch(&P.farflag[v], 1) == 0;
        }
    }
}

template <bool kDelta>
__global__ void k_sssp_relax(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                             const int32_t* __restrict__ w, const int32_t* __restrict__ fq, uint32_t fn,
                             int32_t* __restrict__ dist, int32_t* __restrict__ flag, int32_t* __restrict__ nq,
                             uint32_t* __restrict__ nn, int32_t* __restrict__ hq, uint32_t* __restrict__ hn,
                             SsspPush P) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = warp; i < fn; i += nwarps) {
        const int32_t u = fq[i];
        const uint64_t b = off[u], e = off[u + 1];
        if (e - b > kHeavyDeg) {  // relaxed by k_sssp_relax_heavy
            if (lane == 0) hq[atomicAdd(hn, 1u)] = u;
            continue;
        }
        const int32_t du = dist[u];
        for (uint64_t j0 = b; j0 < e; j0 += 32) {
            const uint64_t j = j0 + lane;
            bool near = false, far = false;
            int32_t v = 0;
            if (j < e) {
                v = adj[j];
                sssp_relax_edge<kDelta>(du, v, w[j], dist, flag, P, &near, &far);
            }
            warp_append(near, v, nq, nn);
            if (kDelta) warp_append(far, v, P.far, P.farn);
        }
    }
}

// The heavy frontier vertices of a relaxation round, spread over the grid.
// dist[u] may fall further while its row is being relaxed; any value read is
// an achieved distance, and a vertex whose distance falls is queued again.
template <bool kDelta>
__global__ void k_sssp_relax_heavy(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                                   const int32_t* __restrict__ w, const int32_t* __restrict__ hq,
                                   const uint32_t* __restrict__ hn, int32_t* __restrict__ dist,
                                   int32_t* __restrict__ flag, int32_t* __restrict__ nq, uint32_t* __restrict__ nn,
                                   SsspPush P) {
    heavy_rows(off, hq, *hn, [&](int32_t u, uint64_t j, bool ok) {
        bool near = false, far = false;
        int32_t v = 0;
        if (ok) {
            v = adj[j];
            sssp_relax_edge<kDelta>(dist[u], v, w[j], dist, flag, P, &near, &far);
        }
        warp_append(near, v, nq, nn);
        if (kDelta) warp_append(far, v, P.far, P.farn);
    });
}

// Smallest current distance in the far pile (entries at or above lo; lower
// ones were relaxed in an earlier bucket), so empty buckets are skipped.
__global__ void k_sssp_far_min(const int32_t* __restrict__ far, uint32_t fn, const int32_t* __restrict__ dist,
                               int32_t lo, int32_t* __restrict__ out) {
    int32_t mn = INT_MAX;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < fn; i += gridDim.x * blockDim.x) {
        const int32_t d = dist[far[i]];
        if (d >= lo) mn = min(mn, d);
    }
    for (int o = 16; o; o >>= 1) mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    if ((threadIdx.x & 31) == 0 && mn != INT_MAX) atomicMin(out, mn);
}

// Splits the far pile at the new bucket [lo, hi): entries whose distance
// fell below lo were relaxed when it fell and are dropped; entries in
// [lo, hi) become the near frontier; the rest stay in the far pile.
__global__ void k_sssp_far_split(const int32_t* __restrict__ far, uint32_t fn, const int32_t* __restrict__ dist,
                                 int32_t lo, int32_t hi, int32_t* __restrict__ flag, int32_t* __restrict__ farflag,
                                 int32_t* __restrict__ nq, uint32_t* __restrict__ nn, int32_t* __restrict__ far2,
                                 uint32_t* __restrict__ far2n) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t nr = (fn + 31) & ~31u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += stride) {
        bool near = false, keep = false;
        int32_t v = 0;
        if (i < fn) {
            v = far[i];
            const int32_t d = dist[v];
            keep = d >= hi;
            if (!keep) {
                farflag[v] = 0;
                near = d >= lo && atomicExch(&flag[v], 1) == 0;
            }
        }
        warp_append(near, v, nq, nn);
        warp_append(keep, v, far2, far2n);
    }
}

// Sum of m int32 values (non-negative weights) into *out.
__global__ void k_sum_i32(const int32_t* __restrict__ a, uint64_t m, unsigned long long* __restrict__ out) {
    unsigned long long x = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
        x += (unsigned long long)(uint32_t)a[i];
    x = warp_sum_u64(x);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(out, x);
}

__global__ void k_clear_flags(const int32_t* __restrict__ q, uint32_t qn, int32_t* __restrict__ flag) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < qn) flag[q[i]] = 0;
}

// Hands the ids of adj[b, e) taken by lane gl of a group of L lanes to
// f(ok, id), four per 16-byte load: the loads start at the 16-byte boundary
// at or below b and step by 4 L ids, so one dependent round gives each lane
// four independent gathers; ok is false for the positions of a load outside
// [b, e), which the caller skips.  A load may run up to 3 ids past e, which
// the 64 ids of padding after the last row keep inside the adjacency array.
// The adjacency is read once per sweep, so its loads carry the streaming
// hint (evict first): the gathered vectors keep their L2 lines.
template <int L, class F>
__device__ __forceinline__ void row_ids_vec4(const int32_t* __restrict__ adj, uint64_t b, uint64_t e, int gl,
                                             F&& f) {
    for (uint64_t q = (b & ~3ull) + 4ull * (uint64_t)gl; q < e; q += 4ull * L) {
        const int4 v = __ldcs(reinterpret_cast<const int4*>(adj + q));
        f(q >= b, v.x);
        f(q + 1 >= b && q + 1 < e, v.y);
        f(q + 2 >= b && q + 2 < e, v.z);
        f(q + 3 < e, v.w);
    }
}

// ---- PageRank (pull) -----------------------------------------------------------

template <class T>
__global__ void k_pr_init(const uint64_t* __restrict__ off, uint64_t n, T damping, const T* __restrict__ init,
                          T* __restrict__ degs, T* __restrict__ contrib) {
    uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (u >= n) return;
    // degs[u] = d(u) / damping; x0 = degs / n (src/Graph.cpp:1563-1570)
    const T dg = (T)(off[u + 1] - off[u]) / damping;
    degs[u] = dg;
    const T x0 = init ? init[u] : dg / (T)n;
    contrib[u] = dg > (T)0 ? x0 / dg : (T)0;
}

// One iteration: x'[v] = base + sum_{u in N(v)} contrib[u]; contrib'[v] = x'[v] / degs[v].
// T is the storage type of the vectors; the row sums, x' and the division
// run in fp64 for both instances, so the fp32 vectors carry only their own
// storage rounding (within 1e-6 relative of the FP64 recurrence at 20
// iterations; fp32 row sums over hub in-lists drift past that).
template <class T>
__device__ __forceinline__ void pr_epilogue(uint64_t v, double base, double sum, const T* __restrict__ degs,
                                            T* __restrict__ x_out, T* __restrict__ contrib_out) {
    const double x = base + sum;
    x_out[v] = (T)x;
    const double dg = (double)degs[v];
    contrib_out[v] = dg > 0.0 ? (T)(x / dg) : (T)0;
}

// One iteration: x'[v] = base + sum_{u in N(v)} contrib[u]; contrib'[v] = x'[v] / degs[v].
// T is the storage type of the vectors; the row sums, x' and the division
// run in fp64 for both instances, so the fp32 vectors carry only their own
// storage rounding (within 1e-6 relative of the FP64 recurrence at 20
// iterations; fp32 row sums over hub in-lists drift past that).  Rows listed
// in hq (more than kPullHeavyDeg entries) get a whole CTA each; the others
// kPullLanes lanes.  Both reductions run in a fixed order, so results are
// reproducible.
template <class T>
__global__ void __launch_bounds__(kThreads) k_pr_iter(const uint64_t* __restrict__ off,
                                                      const int32_t* __restrict__ adj, uint64_t n, double base,
                                                      const T* __restrict__ degs, const T* __restrict__ contrib,
                                                      T* __restrict__ x_out, T* __restrict__ contrib_out,
                                                      const int32_t* __restrict__ hq, uint32_t hn) {
    __shared__ double s_part[kThreads / 32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    for (uint32_t h = blockIdx.x; h < hn; h += gridDim.x) {
        const int32_t v = hq[h];
        const uint64_t b = off[v], e = off[v + 1];
        double s = 0.0;
        row_ids_vec4<kThreads>(adj, b, e, threadIdx.x, [&](bool ok, int32_t u) {
            if (ok) s += (double)__ldg(contrib + u);
        });
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) s_part[wib] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int i = 0; i < kThreads / 32; ++i) t += s_part[i];
            pr_epilogue(v, base, t, degs, x_out, contrib_out);
        }
        __syncthreads();
    }
    // the other rows: kPullLanes lanes each, 32 / kPullLanes rows per warp at once
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    constexpr int kRows = 32 / kPullLanes;
    const int g = lane / kPullLanes, gl = lane % kPullLanes;
    for (uint64_t v0 = warp * kRows; v0 < n; v0 += nwarps * kRows) {
        const uint64_t v = v0 + g;
        uint64_t b = 0, e = 0;
        if (v < n) {
            b = off[v];
            e = off[v + 1];
            if (e - b > kPullHeavyDeg) e = b;  // a CTA row
        }
        double s = 0.0;
        row_ids_vec4<kPullLanes>(adj, b, e, gl, [&](bool ok, int32_t u) {
            if (ok) s += (double)__ldg(contrib + u);
        });
        for (int o = kPullLanes / 2; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (v < n && gl == 0 && off[v + 1] - off[v] <= kPullHeavyDeg) pr_epilogue(v, base, s, degs, x_out, contrib_out);
    }
}

// ---- k-core ----------------------------------------------------------------------

__global__ void k_kcore_init(const uint64_t* __restrict__ off, uint64_t n, int32_t* __restrict__ deg,
                             int32_t* __restrict__ core, int32_t* __restrict__ rem) {
    uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (u >= n) return;
    deg[u] = (int32_t)(off[u + 1] - off[u]);
    core[u] = -1;
    rem[u] = (int32_t)u;
}

// Device-driven peeling in one persistent kernel.  Each step is a peel round
// at the current level when the frontier is not empty, else the scan of the
// next level; a grid barrier separates steps.  The state lives in three
// rotating records: step i reads S[i % 3], accumulates into S[(i+1) % 3]
// (counters cleared by step i-1) and clears S[(i+2) % 3], which no CTA reads
// during step i.  Mutable arrays are read with __ldcg: L1 is not coherent
// across CTAs within one launch.  Frontier vertices with more than kHeavyDeg
// neighbours are set aside (hq0/hq1 by step parity) and their rows are peeled
// in the next step, spread over the grid; that step is still a peel round of
// the same level, so every decrement of a level lands before its next scan.
struct KState {
    int32_t k;      // level of the step that wrote this record
    uint32_t fn;    // frontier size it produced
    uint32_t rn;    // remaining (unpeeled) vertices after it
    int32_t ml;     // minimum degree left (scan steps)
    int32_t phase;  // 0 scan, 1 peel
    int32_t fpar;   // frontier buffer holding the frontier
    int32_t rpar;   // remaining-list buffer
    uint32_t hn;    // heavy frontier vertices it set aside for the next step
};

__device__ __forceinline__ KState load_state(const KState* p) {
    const int4 lo = __ldcg(reinterpret_cast<const int4*>(p));
    const int4 hi = __ldcg(reinterpret_cast<const int4*>(p) + 1);
    KState s;
    s.k = lo.x;
    s.fn = (uint32_t)lo.y;
    s.rn = (uint32_t)lo.z;
    s.ml = lo.w;
    s.phase = hi.x;
    s.fpar = hi.y;
    s.rpar = hi.z;
    s.hn = (uint32_t)hi.w;
    return s;
}

__global__ void __launch_bounds__(kThreads) k_kcore_persistent(
    const uint64_t* __restrict__ off, const int32_t* __restrict__ adj, uint64_t n, int32_t* deg, int32_t* core,
    int32_t* rem0, int32_t* rem1, int32_t* f0, int32_t* f1, int32_t* hq0, int32_t* hq1, KState* S,
    GridBarrier* gb, uint64_t max_steps, uint64_t limit_ns, uint64_t* steps_done, uint32_t local_edges) {
    // decrements of the lowest ids (the hubs, once ids are degree-ordered)
    // are gathered per CTA in shared memory and applied once per step
    __shared__ int32_t s_dec[kKcoreHubs];
    __shared__ int s_any;
    __shared__ int32_t s_lq[2][kLocalQ];
    __shared__ uint32_t s_lqn[2];  // entries pushed (may exceed kLocalQ: the rest went to the frontier)
    __shared__ uint32_t s_lqe[2];  // row entries of the queued vertices
    for (int i = threadIdx.x; i < kKcoreHubs; i += blockDim.x) s_dec[i] = 0;
    if (threadIdx.x == 0) {
        s_any = 0;
        s_lqn[0] = s_lqn[1] = 0;
        s_lqe[0] = s_lqe[1] = 0;
    }
    __syncthreads();
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    const int lane = threadIdx.x & 31;
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t warp = tid >> 5, nwarps = stride >> 5;
    uint64_t step = 0;
    for (; step < max_steps; ++step) {
        const KState in = load_state(&S[step % 3]);
        KState* out = &S[(step + 1) % 3];
        const bool peel = in.fn > 0 || in.hn > 0;
        const int32_t k = peel ? in.k
                               : ((in.phase == 1 || in.ml == INT_MAX) ? in.k + 1 : max(in.k + 1, in.ml + 1));
        // every CTA reads the same record, so all leave at the same step
        if (!peel && (in.rn == 0 || (uint64_t)k >= n)) break;
        if (lead) {
            KState* clr = &S[(step + 2) % 3];
            clr->fn = 0;
            clr->rn = 0;
            clr->ml = INT_MAX;
            clr->hn = 0;
            if (peel) out->rn = in.rn;  // a peel round keeps the remaining list
            out->k = k;
            out->phase = peel ? 1 : 0;
            out->fpar = peel ? 1 - in.fpar : 0;
            out->rpar = peel ? in.rpar : 1 - in.rpar;
        }
        if (peel) {
            const int32_t* fq = in.fpar ? f1 : f0;
            int32_t* nq = in.fpar ? f0 : f1;
            int32_t* hq_next = (step & 1) ? hq1 : hq0;
            const int32_t* hq_prev = (step & 1) ? hq0 : hq1;
            // A vertex pushed at this level goes to this CTA's local queue
            // (s_lq[wr]) while it has room, else to the next step's frontier;
            // the CTA peels its local queue itself, so a level's cascade
            // takes one step instead of one step per round.
            int wr = 0;
            auto push_v = [&](bool pred, int32_t v) {
                const unsigned m = __ballot_sync(0xffffffffu, pred);
                if (!m) return;
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(&s_lqn[wr], (uint32_t)__popc(m));
                base = __shfl_sync(0xffffffffu, base, 0);
                const uint32_t idx = base + __popc(m & ((1u << lane) - 1u));
                const bool local = pred && idx < kLocalQ;
                uint32_t len = 0;
                if (local) {
                    s_lq[wr][idx] = v;
                    len = (uint32_t)min(off[v + 1] - off[v], (uint64_t)kHeavyDeg + 1);
                }
                for (int o = 16; o; o >>= 1) len += __shfl_xor_sync(0xffffffffu, len, o);
                if (lane == 0 && len) atomicAdd(&s_lqe[wr], len);
                warp_append(pred && !local, v, nq, &out->fn);
            };
            // one CSR entry (u, v) of a peeled vertex u; all lanes call it
            auto peel_entry = [&](uint64_t j, bool ok) {
                bool push = false;
                int32_t v = 0;
                if (ok) {
                    v = adj[j];
                    if (__ldcg(core + v) < 0) {
                        if (v < kKcoreHubs) {
                            atomicAdd(&s_dec[v], 1);
                            s_any = 1;
                        } else {
                            const int32_t old = atomicSub(&deg[v], 1);
                            if (old == k) {
                                push = true;
                                core[v] = k - 1;
                            }
                        }
                    }
                }
                push_v(push, v);
            };
            // the row of a peeled vertex u, by one warp (set aside if heavy)
            auto peel_row = [&](int32_t u) {
                const uint64_t b = off[u], e = off[u + 1];
                if (e - b > kHeavyDeg) {
                    if (lane == 0) hq_next[atomicAdd(&out->hn, 1u)] = u;
                    return;
                }
                for (uint64_t j0 = b; j0 < e; j0 += 32) peel_entry(j0 + lane, j0 + lane < e);
            };
            for (uint64_t i = warp; i < in.fn; i += nwarps) peel_row(__ldcg(fq + i));
            heavy_rows(off, hq_prev, in.hn, [&](int32_t, uint64_t j, bool ok) { peel_entry(j, ok); });
            // drain the local queues; when one runs dry, flush the gathered
            // hub decrements (the one flush that takes a degree from >= k to
            // < k pushes the vertex) and go on until nothing is left
            int rd = 0;
            for (;;) {
                __syncthreads();
                uint32_t cnt = min(s_lqn[rd], (uint32_t)kLocalQ);
                if (cnt == 0) {
                    if (s_any) {
                        wr = rd;
                        for (int i = threadIdx.x; i < kKcoreHubs; i += blockDim.x) {
                            const int32_t c = s_dec[i];
                            bool push = false;
                            if (c) {
                                s_dec[i] = 0;
                                const int32_t old = atomicSub(&deg[i], c);
                                if (old >= k && old - c < k) {
                                    push = true;
                                    core[i] = k - 1;
                                }
                            }
                            push_v(push, i);
                        }
                        __syncthreads();
                        if (threadIdx.x == 0) s_any = 0;
                        __syncthreads();
                        cnt = min(s_lqn[rd], (uint32_t)kLocalQ);
                    }
                    if (cnt == 0) break;
                }
                if (s_lqe[rd] > local_edges) {
                    // too much for one CTA: the next step shares it among all
                    const uint32_t cpad = (cnt + 31) & ~31u;
                    for (uint32_t i = threadIdx.x; i < cpad; i += blockDim.x)
                        warp_append(i < cnt, i < cnt ? s_lq[rd][i] : 0, nq, &out->fn);
                    __syncthreads();
                    if (threadIdx.x == 0) {
                        s_lqn[rd] = 0;
                        s_lqe[rd] = 0;
                    }
                    continue;
                }
                wr = rd ^ 1;
                for (uint32_t i = threadIdx.x >> 5; i < cnt; i += blockDim.x >> 5) peel_row(s_lq[rd][i]);
                __syncthreads();
                if (threadIdx.x == 0) {
                    s_lqn[rd] = 0;
                    s_lqe[rd] = 0;
                }
                rd ^= 1;
            }
            if (threadIdx.x == 0) {
                s_lqn[0] = s_lqn[1] = 0;
                s_lqe[0] = s_lqe[1] = 0;
            }
        } else {
            // scan of level k over the remaining list
            const int32_t* rem = in.rpar ? rem1 : rem0;
            int32_t* rem2 = in.rpar ? rem0 : rem1;
            const uint64_t nr = ((uint64_t)in.rn + 31) & ~(uint64_t)31;
            int32_t mn = INT_MAX;
            for (uint64_t i = tid; i < nr; i += stride) {
                bool pl = false, keep = false;
                int32_t u = 0;
                if (i < in.rn) {
                    u = __ldcg(rem + i);
                    if (__ldcg(core + u) < 0) {
                        const int32_t d = __ldcg(deg + u);
                        if (d < k) {
                            // d counts the unpeeled neighbours: with none,
                            // peeling u would decrement nobody
                            pl = d > 0;
                            core[u] = k - 1;
                        } else {
                            keep = true;
                            mn = min(mn, d);
                        }
                    }
                }
                warp_append(pl, u, f0, &out->fn);
                warp_append(keep, u, rem2, &out->rn);
            }
            for (int o = 16; o; o >>= 1) mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
            if (lane == 0 && mn != INT_MAX) atomicMin(&out->ml, mn);
        }
        if (!grid_sync(gb, limit_ns)) return;
    }
    if (lead) {
        *steps_done = step;
        if (step == max_steps) atomicExch(&gb->err, 2);
    }
}

// Self-test of the grid barrier: `rounds` barriers, each CTA adding 1 to
// `tally` before each; CTA `absent` (if >= 0) never arrives, so the others'
// waits run out after limit_ns and the barrier reports it.
__global__ void k_grid_sync_selftest(GridBarrier* gb, int rounds, int absent, uint64_t limit_ns,
                                     unsigned* tally, unsigned* bad) {
    if ((int)blockIdx.x == absent) return;
    for (int r = 0; r < rounds; ++r) {
        if (threadIdx.x == 0) atomicAdd(tally, 1u);
        if (!grid_sync(gb, limit_ns)) return;
        // after barrier r every CTA has added its r+1 increments
        if (threadIdx.x == 0 && __ldcg(tally) < (unsigned)(r + 1) * gridDim.x) atomicAdd(bad, 1u);
        if (!grid_sync(gb, limit_ns)) return;
    }
}

// Vertices never peeled get core 0; *top receives the largest core number.
__global__ void k_kcore_finish(int32_t* __restrict__ core, uint64_t n, int32_t* __restrict__ top) {
    const uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    int32_t c = 0;
    if (u < n) {
        c = core[u];
        if (c < 0) core[u] = c = 0;
    }
    for (int o = 16; o; o >>= 1) c = max(c, __shfl_xor_sync(0xffffffffu, c, o));
    if ((threadIdx.x & 31) == 0 && c > 0) atomicMax(top, c);
}

// ---- MIS -------------------------------------------------------------------------

// Round over the undecided list: OUT if a neighbour is IN; IN if every
// neighbour of smaller priority is OUT; otherwise undecided again.  Decisions
// are final and only made from final neighbour states, so the in-place update
// reaches the unique greedy (lexicographically-first) set.
__global__ void k_mis_round(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                            const uint64_t* __restrict__ prio, const uint32_t* __restrict__ dplus,
                            const int32_t* __restrict__ uq, uint32_t un, int32_t* __restrict__ state,
                            int32_t* __restrict__ nq, uint32_t* __restrict__ nn) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    if (dplus) {
        // With id priorities only the neighbours below u matter: an IN
        // neighbour v > u would need u OUT first, and only v < u block (rows
        // are sorted, so those are the first dplus[u] entries).  Those lists
        // are short, so kMisLanes lanes take a vertex, 32 / kMisLanes at once.
        constexpr int kRows = 32 / kMisLanes;
        const int g = lane / kMisLanes, gl = lane % kMisLanes;
        const unsigned gm = ((1u << kMisLanes) - 1u) << (g * kMisLanes);
        for (uint64_t i0 = warp * kRows; i0 < un; i0 += nwarps * kRows) {
            const uint64_t i = i0 + g;
            const bool have = i < un;
            int32_t u = 0;
            uint64_t b = 0, e = 0;
            if (have) {
                u = uq[i];
                b = off[u];
                e = b + dplus[u];
            }
            bool in_nbr = false, blocked = false;
            for (uint64_t k = 0;; k += kMisLanes) {
                const uint64_t j = b + k + gl;
                bool a = false, c = false;
                if (have && !in_nbr && j < e) {
                    const int32_t v = adj[j];
                    const int32_t sv = state[v];
                    a = sv == 1;
                    c = sv == 0;  // every v here is below u
                }
                // every lane votes (a short-circuit here would skip the
                // vote on some lanes and leave the others waiting)
                const unsigned va = __ballot_sync(0xffffffffu, a);
                const unsigned vc = __ballot_sync(0xffffffffu, c);
                in_nbr = in_nbr || (va & gm) != 0;
                blocked = blocked || (vc & gm) != 0;
                const bool more = have && !in_nbr && b + k + kMisLanes < e;
                if (!__any_sync(0xffffffffu, more)) break;
            }
            if (have && gl == 0) {
                if (in_nbr) state[u] = 2;
                else if (!blocked) state[u] = 1;
            }
            warp_append(have && gl == 0 && !in_nbr && blocked, u, nq, nn);
        }
        return;
    }
    for (uint64_t i = warp; i < un; i += nwarps) {
        const int32_t u = uq[i];
        const uint64_t pu = prio ? prio[u] : (uint64_t)u;
        const uint64_t b = off[u], e = off[u + 1];
        bool in_nbr = false, blocked = false;
        for (uint64_t j0 = b; j0 < e; j0 += 32) {
            const uint64_t j = j0 + lane;
            bool a = false, c = false;
            if (j < e) {
                const int32_t v = adj[j];
                const int32_t sv = state[v];
                a = sv == 1;
                const uint64_t pv = prio ? prio[v] : (uint64_t)v;
                c = sv == 0 && (pv < pu || (pv == pu && v < u));
            }
            in_nbr = __any_sync(0xffffffffu, a) || in_nbr;
            blocked = __any_sync(0xffffffffu, c) || blocked;
            if (in_nbr) break;
        }
        if (lane == 0) {
            if (in_nbr) state[u] = 2;
            else if (!blocked) state[u] = 1;
        }
        const bool again = !in_nbr && blocked;
        if (lane == 0 && again) nq[atomicAdd(nn, 1u)] = u;
    }
}

__global__ void k_mis_prio(uint64_t n, const int32_t* __restrict__ int2api, uint64_t key, int hashed,
                           uint64_t* __restrict__ prio) {
    uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (u >= n) return;
    const uint32_t api = int2api ? (uint32_t)int2api[u] : (uint32_t)u;
    prio[u] = hashed ? pc_vertex_priority(key, api) : (uint64_t)api;
}

__global__ void k_mis_finish(const int32_t* __restrict__ state, uint64_t n, int32_t* __restrict__ res) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) res[i] = state[i] == 1 ? 1 : 0;
}

// ---- CDLP --------------------------------------------------------------------------

// One iteration: out[v] = max label over N(v), 0 for an isolated vertex
// (src/Graph.cpp:650: labels start at 0 for every vertex).  Rows listed in hq
// get a whole CTA each; the others kPullLanes lanes.
__global__ void __launch_bounds__(kThreads) k_cdlp_iter(const uint64_t* __restrict__ off,
                                                        const int32_t* __restrict__ adj, uint64_t n,
                                                        const int32_t* __restrict__ lab, int32_t* __restrict__ out,
                                                        const int32_t* __restrict__ hq, uint32_t hn) {
    __shared__ int32_t s_part[kThreads / 32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    for (uint32_t h = blockIdx.x; h < hn; h += gridDim.x) {
        const int32_t v = hq[h];
        const uint64_t b = off[v], e = off[v + 1];
        int32_t mx = 0;
        row_ids_vec4<kThreads>(adj, b, e, threadIdx.x, [&](bool ok, int32_t u) {
            if (ok) mx = max(mx, __ldg(lab + u));
        });
        for (int o = 16; o; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (lane == 0) s_part[wib] = mx;
        __syncthreads();
        if (threadIdx.x == 0) {
            int32_t t = 0;
            for (int i = 0; i < kThreads / 32; ++i) t = max(t, s_part[i]);
            out[v] = t;
        }
        __syncthreads();
    }
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    constexpr int kRows = 32 / kPullLanes;
    const int g = lane / kPullLanes, gl = lane % kPullLanes;
    for (uint64_t v0 = warp * kRows; v0 < n; v0 += nwarps * kRows) {
        const uint64_t v = v0 + g;
        uint64_t b = 0, e = 0;
        if (v < n) {
            b = off[v];
            e = off[v + 1];
            if (e - b > kPullHeavyDeg) e = b;  // a CTA row
        }
        int32_t mx = 0;
        row_ids_vec4<kPullLanes>(adj, b, e, gl, [&](bool ok, int32_t u) {
            if (ok) mx = max(mx, __ldg(lab + u));
        });
        for (int o = kPullLanes / 2; o; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (v < n && gl == 0 && off[v + 1] - off[v] <= kPullHeavyDeg) out[v] = mx;
    }
}

}  // namespace fr

using namespace fr;

static unsigned grid_for(const pc_pgraph* pg, int per_sm = 8) { return (unsigned)(sm_count(pg->g->device) * per_sm); }

// Entries a heavy list can need: rows of more than kHeavyDeg entries.
static uint64_t heavy_cap(uint64_t n, uint64_t m) { return std::max<uint64_t>(1, std::min<uint64_t>(n, m / kHeavyDeg + 1)); }
static uint64_t pull_heavy_cap(uint64_t n, uint64_t m) {
    return std::max<uint64_t>(1, std::min<uint64_t>(n, m / kPullHeavyDeg + 1));
}

// Lists the rows of more than kPullHeavyDeg entries into hq (room for
// pull_heavy_cap entries) and reads their number back.
static pc_status list_heavy_rows(pc_pgraph* pg, int32_t* hq, uint32_t* d_hn, uint32_t* hn) {
    if (!hq || !d_hn) return fail(PC_ERR_OOM, "scratch plan exceeds its reservation");
    cudaStream_t s = pg->g->stream;
    PC_CUDA(cudaMemsetAsync(d_hn, 0, 4, s));
    k_heavy_list<<<grid_for(pg), kThreads, 0, s>>>(pg->off, pg->g->n, kPullHeavyDeg, hq, d_hn);
    PC_LAUNCHED();
    PC_CUDA(cudaMemcpyAsync(hn, d_hn, 4, cudaMemcpyDeviceToHost, s));
    PC_CUDA(cudaStreamSynchronize(s));
    return PC_OK;
}

// Reads a device counter (synchronising the stream).
static pc_status read_u32(pc_pgraph* pg, const uint32_t* d, uint32_t* h) {
    PC_CUDA(cudaMemcpyAsync(h, d, 4, cudaMemcpyDeviceToHost, pg->g->stream));
    PC_CUDA(cudaStreamSynchronize(pg->g->stream));
    return PC_OK;
}

static pc_status bfs_run(pc_pgraph* pg, int32_t src, int32_t* rank_host) {
    const uint64_t n = pg->g->n, m = pg->g->m;
    cudaStream_t s = pg->g->stream;
    const uint64_t hcap = heavy_cap(n, m);
    PC_TRY(scratch_reserve(pg, n * 4 * 4 + hcap * 4 + 256));
    int32_t* dist = pg->scratch.take<int32_t>(n);
    int32_t* q0 = pg->scratch.take<int32_t>(n);
    int32_t* q1 = pg->scratch.take<int32_t>(n);
    int32_t* hq = pg->scratch.take<int32_t>(hcap);
    uint32_t* cnt = pg->scratch.take<uint32_t>(4);  // [0] next frontier, [1] heavy list
    unsigned long long* edges = pg->scratch.take<unsigned long long>(2);
    if (!edges) return fail(PC_ERR_OOM, "BFS scratch plan exceeds its reservation");
    const unsigned nb = (unsigned)ceil_div(n, kThreads);
    k_fill_i32<<<nb, kThreads, 0, s>>>(dist, n, kInf);
    PC_LAUNCHED();
    const int32_t zero = 0;
    PC_CUDA(cudaMemcpyAsync(dist + src, &zero, 4, cudaMemcpyHostToDevice, s));
    PC_CUDA(cudaMemcpyAsync(q0, &src, 4, cudaMemcpyHostToDevice, s));
    // host-side state of the direction heuristic (Beamer, Asanovic, Patterson, SC'12)
    std::vector<uint64_t> h_off(2);
    PC_CUDA(cudaMemcpyAsync(h_off.data(), pg->off + src, 16, cudaMemcpyDeviceToHost, s));
    PC_CUDA(cudaStreamSynchronize(s));
    uint64_t frontier_edges = h_off[1] - h_off[0];
    uint64_t unexplored = m - frontier_edges;
    uint32_t fn = 1;
    bool bottom_up = false;
    const double alpha = 15.0, beta = 18.0;
    int32_t* fq = q0;
    int32_t* nq = q1;
    for (int32_t level = 1; fn > 0; ++level) {
        if (!bottom_up && (double)frontier_edges > (double)unexplored / alpha) bottom_up = true;
        else if (bottom_up && (double)fn < (double)n / beta) bottom_up = false;
        PC_CUDA(cudaMemsetAsync(cnt, 0, 8, s));
        PC_CUDA(cudaMemsetAsync(edges, 0, 8, s));
        if (bottom_up) {
            k_bfs_bottom_up<<<grid_for(pg), kThreads, 0, s>>>(pg->off, pg->adj, n, dist, level, nq, cnt, edges);
        } else {
            k_bfs_top_down<<<grid_for(pg), kThreads, 0, s>>>(pg->off, pg->adj, fq, fn, dist, level, nq, cnt, edges,
                                                             hq, cnt + 1);
            PC_LAUNCHED();
            k_bfs_top_down_heavy<<<grid_for(pg), kThreads, 0, s>>>(pg->off, pg->adj, hq, cnt + 1, dist, level, nq, cnt,
                                                                   edges);
        }
        PC_LAUNCHED();
        unsigned long long h_edges = 0;
        PC_CUDA(cudaMemcpyAsync(&fn, cnt, 4, cudaMemcpyDeviceToHost, s));
        PC_CUDA(cudaMemcpyAsync(&h_edges, edges, 8, cudaMemcpyDeviceToHost, s));
        PC_CUDA(cudaStreamSynchronize(s));
        frontier_edges = h_edges;
        unexplored = unexplored > h_edges ? unexplored - h_edges : 0;
        std::swap(fq, nq);
        if (level > (int32_t)n + 1) return fail(PC_ERR_TIMEOUT, "BFS did not converge");
    }
    int32_t* rank_int = q0 == fq ? q1 : q0;  // any free n-array
    k_bfs_finish<<<nb, kThreads, 0, s>>>(dist, n, rank_int);
    PC_LAUNCHED();
    int32_t* rank_api = dist;
    PC_TRY(gather_to_api_i32(pg, rank_int, rank_api));
    PC_CUDA(cudaMemcpyAsync(rank_host, rank_api, n * 4, cudaMemcpyDeviceToHost, s));
    return sync(pg);
}

template <class T>
static pc_status pagerank_run(pc_pgraph* pg, T damping, int32_t iters, const T* init, T* out_host) {
    const uint64_t n = pg->g->n;
    cudaStream_t s = pg->g->stream;
    const uint64_t hcap = pull_heavy_cap(n, pg->g->m);
    PC_TRY(scratch_reserve(pg, n * sizeof(T) * 6 + hcap * 4 + 512));
    int32_t* hq = pg->scratch.take<int32_t>(hcap);
    uint32_t* d_hn = pg->scratch.take<uint32_t>(1);
    T* degs = pg->scratch.take<T>(n);
    T* c0 = pg->scratch.take<T>(n);
    T* c1 = pg->scratch.take<T>(n);
    T* x = pg->scratch.take<T>(n);
    T* xapi = pg->scratch.take<T>(n);
    T* ini = nullptr;
    const unsigned nb = (unsigned)ceil_div(n, kThreads);
    if (init) {
        ini = pg->scratch.take<T>(n);
        PC_CUDA(cudaMemcpyAsync(xapi, init, n * sizeof(T), cudaMemcpyHostToDevice, s));
        if (sizeof(T) == 4) PC_TRY(gather_to_internal_f32(pg, (const float*)xapi, (float*)ini));
        else PC_TRY(gather_to_internal_f64(pg, (const double*)xapi, (double*)ini));
    }
    k_pr_init<T><<<nb, kThreads, 0, s>>>(pg->off, n, damping, ini, degs, c0);
    PC_LAUNCHED();
    uint32_t hn = 0;
    PC_TRY(list_heavy_rows(pg, hq, d_hn, &hn));
    // (1 - damping) / n (src/Graph.cpp:1558), in fp64 like the row sums
    const double base = (1.0 - (double)damping) / (double)n;
    for (int32_t it = 0; it < iters; ++it) {
        k_pr_iter<T><<<grid_for(pg, 16), kThreads, 0, s>>>(pg->off, pg->adj, n, base, degs, c0, x, c1, hq, hn);
        PC_LAUNCHED();
        std::swap(c0, c1);
    }
    if (sizeof(T) == 4) PC_TRY(gather_to_api_f32(pg, (const float*)x, (float*)xapi));
    else PC_TRY(gather_to_api_f64(pg, (const double*)x, (double*)xapi));
    PC_CUDA(cudaMemcpyAsync(out_host, xapi, n * sizeof(T), cudaMemcpyDeviceToHost, s));
    return sync(pg);
}

static pc_status mis_run(pc_pgraph* pg, bool hashed, uint64_t seed, int32_t* res_host) {
    const uint64_t n = pg->g->n;
    cudaStream_t s = pg->g->stream;
    PC_TRY(scratch_reserve(pg, n * 4 * 4 + n * 8 + 256));
    int32_t* state = pg->scratch.take<int32_t>(n);
    int32_t* q0 = pg->scratch.take<int32_t>(n);
    int32_t* q1 = pg->scratch.take<int32_t>(n);
    int32_t* out = pg->scratch.take<int32_t>(n);
    uint64_t* prio = nullptr;
    uint32_t* cnt = pg->scratch.take<uint32_t>(2);
    const unsigned nb = (unsigned)ceil_div(n, kThreads);
    const int32_t* int2api = api_is_internal(pg) ? nullptr : pg->old2new.as<int32_t>();
    if (hashed || int2api) {
        prio = pg->scratch.take<uint64_t>(n);
        k_mis_prio<<<nb, kThreads, 0, s>>>(n, int2api, pc_graph_key(seed, PC_GEN_PRIORITY), hashed ? 1 : 0, prio);
        PC_LAUNCHED();
    }
    const uint32_t* dp = nullptr;
    if (!prio) {
        PC_TRY(ensure_dplus(pg));
        dp = pg->dplus.as<uint32_t>();
    }
    PC_CUDA(cudaMemsetAsync(state, 0, n * 4, s));
    // all vertices start undecided
    k_iota<<<nb, kThreads, 0, s>>>(q0, n);
    PC_LAUNCHED();
    uint32_t un = (uint32_t)n;
    int32_t* fq = q0;
    int32_t* nq = q1;
    for (uint64_t round = 0; un > 0; ++round) {
        PC_CUDA(cudaMemsetAsync(cnt, 0, 4, s));
        k_mis_round<<<grid_for(pg), kThreads, 0, s>>>(pg->off, pg->adj, prio, dp, fq, un, state, nq, cnt);
        PC_LAUNCHED();
        PC_TRY(read_u32(pg, cnt, &un));
        std::swap(fq, nq);
        if (round > n + 1) return fail(PC_ERR_TIMEOUT, "MIS did not converge");
    }
    k_mis_finish<<<nb, kThreads, 0, s>>>(state, n, q0);
    PC_LAUNCHED();
    PC_TRY(gather_to_api_i32(pg, q0, out));
    PC_CUDA(cudaMemcpyAsync(res_host, out, n * 4, cudaMemcpyDeviceToHost, s));
    return sync(pg);
}

}  // namespace pc

using namespace pc;

extern "C" {

pc_status pc_bfs(pc_pgraph* pg, int32_t src, int32_t* rank) {
    clear_error();
    if (!pg || !rank) return fail(PC_ERR_INVALID_INPUT, "null argument");
    const uint64_t n = pg->g->n;
    if (src < 0 || (uint64_t)src >= n) return fail(PC_ERR_INVALID_INPUT, "source vertex out of range");
    PC_TRY(use_device(pg->g));
    return bfs_run(pg, to_internal_id(pg, src), rank);
}

pc_status pc_sssp(pc_pgraph* pg, int32_t src, int32_t* dist_host) {
    return pc_sssp_ex(pg, src, PC_SSSP_AUTO, 0, dist_host);
}

pc_status pc_sssp_ex(pc_pgraph* pg, int32_t src, int32_t method, int32_t delta, int32_t* dist_host) {
    clear_error();
    if (!pg || !dist_host) return fail(PC_ERR_INVALID_INPUT, "null argument");
    const uint64_t n = pg->g->n, m = pg->g->m;
    if (!pg->w) return fail(PC_ERR_INVALID_INPUT, "SSSP needs a weighted graph");
    if (src < 0 || (uint64_t)src >= n) return fail(PC_ERR_INVALID_INPUT, "source vertex out of range");
    if (method != PC_SSSP_AUTO && method != PC_SSSP_BELLMAN_FORD && method != PC_SSSP_DELTA_STEPPING)
        return fail(PC_ERR_INVALID_INPUT, "unknown SSSP method");
    if (delta < 0) return fail(PC_ERR_INVALID_INPUT, "delta must be >= 0 (0: chosen from the graph)");
    PC_TRY(use_device(pg->g));
    const bool use_delta = method != PC_SSSP_BELLMAN_FORD;
    const int32_t isrc = to_internal_id(pg, src);
    cudaStream_t s = pg->g->stream;
    const uint64_t hcap = heavy_cap(n, m);
    PC_TRY(scratch_reserve(pg, n * 4 * (use_delta ? 9 : 5) + hcap * 4 + 1024));
    int32_t* dist = pg->scratch.take<int32_t>(n);
    int32_t* flag = pg->scratch.take<int32_t>(n);
    int32_t* q0 = pg->scratch.take<int32_t>(n);
    int32_t* q1 = pg->scratch.take<int32_t>(n);
    int32_t* out = pg->scratch.take<int32_t>(n);
    int32_t* hq = pg->scratch.take<int32_t>(hcap);
    uint32_t* cnt = pg->scratch.take<uint32_t>(8);  // [0] next frontier, [1] heavy list, [2] far, [3] far', [4] min
    int32_t *farflag = nullptr, *far0 = nullptr, *far1 = nullptr;
    unsigned long long* wsum = nullptr;
    if (use_delta) {
        farflag = pg->scratch.take<int32_t>(n);
        far0 = pg->scratch.take<int32_t>(n);
        far1 = pg->scratch.take<int32_t>(n);
        wsum = pg->scratch.take<unsigned long long>(1);
    }
    if (!cnt || (use_delta && !wsum)) return fail(PC_ERR_OOM, "SSSP scratch plan exceeds its reservation");
    const unsigned nb = (unsigned)ceil_div(n, kThreads);
    k_fill_i32<<<nb, kThreads, 0, s>>>(dist, n, INT_MAX / 2);  // src/test.cpp:202-203
    PC_LAUNCHED();
    PC_CUDA(cudaMemsetAsync(flag, 0, n * 4, s));
    PC_CUDA(cudaMemsetAsync(cnt, 0, 32, s));
    int32_t bucket = INT_MAX;  // Bellman-Ford: one unbounded bucket
    if (use_delta) {
        PC_CUDA(cudaMemsetAsync(farflag, 0, n * 4, s));
        if (delta == 0) {
            // Delta = 8 x mean weight.  Each relaxation round costs a launch and
            // a host read of the queue size, so narrow buckets (many rounds per
            // bucket) lose: on RMAT-22/24 with weights 1..255 the width of
            // 32 x mean weight / mean degree (134; Davidson et al.) ran 1.3x
            // slower than Bellman-Ford, while widths of 1024 and above ran 1-2 %
            // faster than it.
            PC_CUDA(cudaMemsetAsync(wsum, 0, 8, s));
            k_sum_i32<<<grid_for(pg), kThreads, 0, s>>>(pg->w, m, wsum);
            PC_LAUNCHED();
            unsigned long long h = 0;
            PC_CUDA(cudaMemcpyAsync(&h, wsum, 8, cudaMemcpyDeviceToHost, s));
            PC_TRY(sync(pg));
            const double mean_w = m ? (double)h / (double)m : 1.0;
            delta = (int32_t)std::min<double>(1 << 30, std::max(1.0, std::round(8.0 * mean_w)));
        }
        bucket = delta;
    }
    const int32_t zero = 0;
    PC_CUDA(cudaMemcpyAsync(dist + isrc, &zero, 4, cudaMemcpyHostToDevice, s));
    PC_CUDA(cudaMemcpyAsync(q0, &isrc, 4, cudaMemcpyHostToDevice, s));
    uint32_t fn = 1, farn = 0;
    int32_t* fq = q0;
    int32_t* nq = q1;
    int32_t thr = bucket;
    uint64_t rounds = 0;
    const uint64_t round_cap = 4 * (n + 1) + 64;
    for (;;) {
        while (fn > 0) {
            PC_CUDA(cudaMemsetAsync(cnt, 0, 8, s));
            SsspPush P{thr, far0, cnt + 2, farflag};
            if (use_delta) {
                k_sssp_relax<true><<<grid_for(pg), kThreads, 0, s>>>(pg->off, pg->adj, pg->w, fq, fn, dist, flag, nq,
                                                                    cnt, hq, cnt + 1, P);
                PC_LAUNCHED();
                k_sssp_relax_heavy<true><<<grid_for(pg), kThreads, 0, s>>>(pg->off, pg->adj, pg->w, hq, cnt + 1, dist,
                                                                          flag, nq, cnt, P);
            } else {
                k_sssp_relax<false><<<grid_for(pg), kThreads, 0, s>>>(pg->off, pg->adj, pg->w, fq, fn, dist, flag,
                                                                     nq, cnt, hq, cnt + 1, P);
                PC_LAUNCHED();
                k_sssp_relax_heavy<false><<<grid_for(pg), kThreads, 0, s>>>(pg->off, pg->adj, pg->w, hq, cnt + 1,
                                                                           dist, flag, nq, cnt, P);
            }
            PC_LAUNCHED();
            PC_TRY(read_u32(pg, cnt, &fn));
            if (fn) {
                k_clear_flags<<<(unsigned)ceil_div(fn, kThreads), kThreads, 0, s>>>(nq, fn, flag);
                PC_LAUNCHED();
            }
            std::swap(fq, nq);
            if (++rounds > round_cap) return fail(PC_ERR_TIMEOUT, "SSSP did not converge");
        }
        if (!use_delta) break;
        PC_TRY(read_u32(pg, cnt + 2, &farn));
        if (farn == 0) break;
        // next bucket: from the smallest far distance at or above thr (the
        // entries below thr were relaxed when their distance fell)
        const int32_t big = INT_MAX;
        PC_CUDA(cudaMemcpyAsync(cnt + 4, &big, 4, cudaMemcpyHostToDevice, s));
        k_sssp_far_min<<<(unsigned)std::min<uint64_t>(ceil_div(farn, kThreads), 1024), kThreads, 0, s>>>(
            far0, farn, dist, thr, reinterpret_cast<int32_t*>(cnt + 4));
        PC_LAUNCHED();
        uint32_t mn_u = 0;
        PC_TRY(read_u32(pg, cnt + 4, &mn_u));
        const int32_t mn = (int32_t)mn_u;
        const int32_t lo = thr;
        const int32_t hi = mn == INT_MAX ? INT_MAX : (int32_t)std::min<int64_t>(INT_MAX, (int64_t)mn + delta);
        PC_CUDA(cudaMemsetAsync(cnt, 0, 4, s));
        PC_CUDA(cudaMemsetAsync(cnt + 3, 0, 4, s));
        k_sssp_far_split<<<(unsigned)std::min<uint64_t>(ceil_div(farn, kThreads), 4096), kThreads, 0, s>>>(
            far0, farn, dist, lo, hi, flag, farflag, fq, cnt, far1, cnt + 3);
        PC_LAUNCHED();
        PC_TRY(read_u32(pg, cnt, &fn));
        PC_TRY(read_u32(pg, cnt + 3, &farn));
        if (fn) {
            k_clear_flags<<<(unsigned)ceil_div(fn, kThreads), kThreads, 0, s>>>(fq, fn, flag);
            PC_LAUNCHED();
        }
        std::swap(far0, far1);
        PC_CUDA(cudaMemcpyAsync(cnt + 2, &farn, 4, cudaMemcpyHostToDevice, s));
        thr = hi;
        if (fn == 0 && farn == 0) break;
        if (++rounds > round_cap) return fail(PC_ERR_TIMEOUT, "SSSP did not converge");
    }
    PC_TRY(gather_to_api_i32(pg, dist, out));
    PC_CUDA(cudaMemcpyAsync(dist_host, out, n * 4, cudaMemcpyDeviceToHost, s));
    return sync(pg);
}

pc_status pc_pagerank(pc_pgraph* pg, float damping, int32_t iterations, const float* init, float* out) {
    clear_error();
    if (!pg || !out) return fail(PC_ERR_INVALID_INPUT, "null argument");
    if (iterations <= 0) return fail(PC_ERR_INVALID_INPUT, "iterations must be positive");
    if (!(damping > 0.f && damping <= 1.f)) return fail(PC_ERR_INVALID_INPUT, "damping must be in (0, 1]");
    PC_TRY(use_device(pg->g));
    return pagerank_run<float>(pg, damping, iterations, init, out);
}

pc_status pc_pagerank_f64(pc_pgraph* pg, double damping, int32_t iterations, const double* init, double* out) {
    clear_error();
    if (!pg || !out) return fail(PC_ERR_INVALID_INPUT, "null argument");
    if (iterations <= 0) return fail(PC_ERR_INVALID_INPUT, "iterations must be positive");
    if (!(damping > 0.0 && damping <= 1.0)) return fail(PC_ERR_INVALID_INPUT, "damping must be in (0, 1]");
    PC_TRY(use_device(pg->g));
    return pagerank_run<double>(pg, damping, iterations, init, out);
}

pc_status pc_selftest_grid_barrier(int32_t device, int32_t rounds, int32_t absent_cta, uint32_t limit_ms,
                                   uint32_t* mismatches) {
    clear_error();
    if (rounds < 0 || !mismatches || limit_ms == 0) return fail(PC_ERR_INVALID_INPUT, "bad argument");
    PC_TRY(pc_set_device(device));
    int per_sm = 0;
    PC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_grid_sync_selftest, kThreads, 0));
    if (per_sm < 1) return fail(PC_ERR_CUDA, "self-test kernel cannot be resident");
    const int grid = sm_count(device) * std::min(per_sm, 2);
    if (absent_cta >= grid) return fail(PC_ERR_INVALID_INPUT, "absent_cta is outside the grid");
    cudaStream_t s = nullptr;
    PC_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    DevBuf buf;
    pc_status st = buf.alloc(sizeof(GridBarrier) + 16, "self-test state");
    if (st != PC_OK) {
        cudaStreamDestroy(s);
        return st;
    }
    GridBarrier* gb = buf.as<GridBarrier>();
    unsigned* tally = reinterpret_cast<unsigned*>(gb + 1);
    unsigned* bad = tally + 1;
    uint64_t limit_ns = (uint64_t)limit_ms * 1000000ull;
    void* args[] = {(void*)&gb, (void*)&rounds, (void*)&absent_cta, (void*)&limit_ns, (void*)&tally, (void*)&bad};
    GridBarrier hb{};
    unsigned hbad = 0;
    cudaError_t e = cudaMemsetAsync(buf.p, 0, sizeof(GridBarrier) + 16, s);
    if (e == cudaSuccess)
        e = cudaLaunchCooperativeKernel((const void*)k_grid_sync_selftest, dim3(grid), dim3(kThreads), args, 0, s);
    count_launch();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hb, gb, sizeof(hb), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (e != cudaSuccess) return cuda_fail(e, "grid barrier self-test", __FILE__, __LINE__);
    *mismatches = hbad;
    if (hb.err) return fail(PC_ERR_TIMEOUT, "grid barrier: a wait ran out of time");
    return PC_OK;
}

// Row entries of a CTA's local queue above which the queue goes to the next
// step's frontier (shared by every CTA): kLocalEdges, or PC_KCORE_LOCAL_EDGES
// from the environment (read once; a switch for measurements).
static uint32_t kcore_local_edges() {
    static const uint32_t v = [] {
        const char* e = getenv("PC_KCORE_LOCAL_EDGES");
        const long x = e ? atol(e) : (long)kLocalEdges;
        return (uint32_t)std::max(64L, std::min(x, 1L << 20));
    }();
    return v;
}

pc_status pc_kcore(pc_pgraph* pg, int32_t* core_host, int32_t* largest) {
    clear_error();
    if (!pg || !core_host) return fail(PC_ERR_INVALID_INPUT, "null argument");
    PC_TRY(use_device(pg->g));
    const uint64_t n = pg->g->n;
    cudaStream_t s = pg->g->stream;
    if (n == 0) {
        if (largest) *largest = 0;
        return PC_OK;
    }
    const uint64_t hcap = heavy_cap(n, pg->g->m);
    PC_TRY(scratch_reserve(pg, n * 4 * 7 + hcap * 8 + sizeof(KState) * 3 + sizeof(GridBarrier) + 16));
    int32_t* deg = pg->scratch.take<int32_t>(n);
    int32_t* core = pg->scratch.take<int32_t>(n);
    int32_t* rem0 = pg->scratch.take<int32_t>(n);
    int32_t* rem1 = pg->scratch.take<int32_t>(n);
    int32_t* f0 = pg->scratch.take<int32_t>(n);
    int32_t* f1 = pg->scratch.take<int32_t>(n);
    int32_t* out = pg->scratch.take<int32_t>(n);
    int32_t* hq0 = pg->scratch.take<int32_t>(hcap);
    int32_t* hq1 = pg->scratch.take<int32_t>(hcap);
    KState* S = pg->scratch.take<KState>(3);
    GridBarrier* gb = pg->scratch.take<GridBarrier>(1);
    uint64_t* d_steps = pg->scratch.take<uint64_t>(1);
    int32_t* d_top = pg->scratch.take<int32_t>(1);
    if (!d_top) return fail(PC_ERR_OOM, "k-core scratch plan exceeds its reservation");
    const unsigned nb = (unsigned)ceil_div(n, kThreads);
    k_kcore_init<<<nb, kThreads, 0, s>>>(pg->off, n, deg, core, rem0);
    PC_LAUNCHED();
    // Levels k = 1 .. n-1, as the reference's loop (src/Graph.cpp:683, 1893):
    // at level k every remaining vertex of degree < k gets core k-1, and
    // peeling repeats until no degree crosses below k; empty levels jump to
    // the minimum degree left, as the reference does (src/Graph.cpp:1921).
    // Vertices never peeled (only in a complete graph) keep core 0.
    KState init[3] = {};
    init[0].rn = (uint32_t)n;
    init[1].ml = INT_MAX;
    PC_CUDA(cudaMemcpyAsync(S, init, sizeof(init), cudaMemcpyHostToDevice, s));
    PC_CUDA(cudaMemsetAsync(gb, 0, sizeof(GridBarrier), s));
    PC_CUDA(cudaMemsetAsync(d_top, 0, 4, s));
    int per_sm = 0;
    PC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_kcore_persistent, kThreads, 0));
    if (per_sm < 1) return fail(PC_ERR_CUDA, "k-core kernel cannot be resident");
    const unsigned grid = (unsigned)(sm_count(pg->g->device) * std::min(per_sm, 4));
    // a step scans a level, peels a frontier or peels set-aside heavy rows;
    // each vertex enters a frontier and a heavy list at most once, so n
    // levels plus 2n peel rounds bound the steps
    uint64_t max_steps = 3 * n + 8;
    uint64_t limit_ns = kBarrierLimitNs;
    const uint64_t* off = pg->off;
    const int32_t* adj = pg->adj;
    uint64_t nn = n;
    uint32_t local_edges = kcore_local_edges();
    void* args[] = {(void*)&off,  (void*)&adj, (void*)&nn, (void*)&deg, (void*)&core, (void*)&rem0,
                    (void*)&rem1, (void*)&f0,  (void*)&f1, (void*)&hq0, (void*)&hq1,  (void*)&S,
                    (void*)&gb,   (void*)&max_steps, (void*)&limit_ns, (void*)&d_steps, (void*)&local_edges};
    PC_CUDA(cudaLaunchCooperativeKernel((const void*)k_kcore_persistent, dim3(grid), dim3(kThreads), args, 0, s));
    PC_LAUNCHED();
    k_kcore_finish<<<nb, kThreads, 0, s>>>(core, n, d_top);
    PC_LAUNCHED();
    PC_TRY(gather_to_api_i32(pg, core, out));
    PC_CUDA(cudaMemcpyAsync(core_host, out, n * 4, cudaMemcpyDeviceToHost, s));
    GridBarrier hb{};
    int32_t top = 0;
    PC_CUDA(cudaMemcpyAsync(&hb, gb, sizeof(hb), cudaMemcpyDeviceToHost, s));
    PC_CUDA(cudaMemcpyAsync(&top, d_top, 4, cudaMemcpyDeviceToHost, s));
    PC_TRY(sync(pg));
    // the kernel's own status decides whether core_host holds a result
    if (hb.err == 1) return fail(PC_ERR_TIMEOUT, "k-core: a grid barrier wait ran out of time");
    if (hb.err) return fail(PC_ERR_TIMEOUT, "k-core peeling did not finish within its step bound");
    if (largest) *largest = top;
    return PC_OK;
}

pc_status pc_mis(pc_pgraph* pg, int32_t* res) {
    clear_error();
    if (!pg || !res) return fail(PC_ERR_INVALID_INPUT, "null argument");
    PC_TRY(use_device(pg->g));
    if (pg->g->n == 0) return PC_OK;
    return mis_run(pg, false, 0, res);
}

pc_status pc_mis_hashed(pc_pgraph* pg, uint64_t seed, int32_t* res) {
    clear_error();
    if (!pg || !res) return fail(PC_ERR_INVALID_INPUT, "null argument");
    PC_TRY(use_device(pg->g));
    if (pg->g->n == 0) return PC_OK;
    return mis_run(pg, true, seed, res);
}

pc_status pc_cdlp(pc_pgraph* pg, int32_t iterations, int32_t* labels) {
    clear_error();
    if (!pg || !labels) return fail(PC_ERR_INVALID_INPUT, "null argument");
    if (iterations < 0) return fail(PC_ERR_INVALID_INPUT, "iterations must be non-negative");
    PC_TRY(use_device(pg->g));
    const uint64_t n = pg->g->n;
    if (n == 0 || iterations == 0) return PC_OK;
    cudaStream_t s = pg->g->stream;
    const uint64_t hcap = pull_heavy_cap(n, pg->g->m);
    PC_TRY(scratch_reserve(pg, n * 4 * 3 + hcap * 4 + 512));
    int32_t* a = pg->scratch.take<int32_t>(n);
    int32_t* b = pg->scratch.take<int32_t>(n);
    int32_t* c = pg->scratch.take<int32_t>(n);
    int32_t* hq = pg->scratch.take<int32_t>(hcap);
    uint32_t* d_hn = pg->scratch.take<uint32_t>(1);
    if (!d_hn) return fail(PC_ERR_OOM, "CDLP scratch plan exceeds its reservation");
    PC_CUDA(cudaMemcpyAsync(c, labels, n * 4, cudaMemcpyHostToDevice, s));
    PC_TRY(gather_to_internal_i32(pg, c, a));
    uint32_t hn = 0;
    PC_TRY(list_heavy_rows(pg, hq, d_hn, &hn));
    for (int32_t it = 0; it < iterations; ++it) {
        k_cdlp_iter<<<grid_for(pg, 16), kThreads, 0, s>>>(pg->off, pg->adj, n, a, b, hq, hn);
        PC_LAUNCHED();
        std::swap(a, b);
    }
    PC_TRY(gather_to_api_i32(pg, a, c));
    PC_CUDA(cudaMemcpyAsync(labels, c, n * 4, cudaMemcpyDeviceToHost, s));
    return sync(pg);
}

}  // extern "C"
