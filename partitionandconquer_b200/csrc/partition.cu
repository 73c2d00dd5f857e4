// Greedy vertex partitioning on the GPU: Graph::greedy_partition
// (src/Graph.cpp:898-967) with seeded randomness.
//
// The reference visits vertices by descending degree.  For each vertex u it
// counts its neighbours already placed in each partition, and spreads its
// unplaced neighbours over the partitions: partition i takes
// max(0, deg(u)/P - count_i) / sum * |unplaced| of them (a shuffled list cut
// into consecutive runs); the rest, and every vertex never reached, get a
// random partition.  When deg(u) < P every quota is zero, so all of u's
// unplaced neighbours are placed at random; only the "heavy" vertices
// (deg >= P), which come first in the order, place anything by quota.
//
// GPU form.  Sort by (descending degree, ascending id).  The heavy vertices
// run in waves of kWave consecutive ranks, one CTA each, two launches per
// wave: (1) every wave vertex claims its unplaced neighbours with atomicMin
// of its rank, so a neighbour goes to the earliest vertex that sees it, as in
// the sequential order; (2) every wave vertex counts its neighbours placed
// before the wave (shared-memory counters, one per partition), computes the
// quotas, and places its claimed neighbours: the k-th claimed neighbour (in
// row order, by a block scan) goes to position perm(k) of a seeded affine
// permutation of [0, F), and the position picks the partition whose run holds
// it.  Finally every vertex still unplaced gets a seeded random partition.
// Within a wave a vertex does not see what the others place in the same wave;
// that is the only difference from the sequential rule.
#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <vector>

#include "pc_internal.cuh"
#include "synth_rng.h"

namespace pc {
namespace part {

constexpr int kThreads = 256;
constexpr int kWave = 64;           // heavy vertices per wave
constexpr int kMaxParts = 16384;    // shared-memory counters (8 B each, 128 KB)

__global__ void k_degree_order_keys(const uint64_t* __restrict__ off, uint64_t n, uint64_t* __restrict__ keys) {
    const uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (u < n) keys[u] = ((0xFFFFFFFFull - (off[u + 1] - off[u])) << 32) | u;
}

// order[r] = vertex of rank r; *heavy = number of ranks with degree >= P.
__global__ void k_order(const uint64_t* __restrict__ keys, uint64_t n, uint32_t P, int32_t* __restrict__ order,
                        uint32_t* __restrict__ heavy) {
    const uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    order[r] = (int32_t)(keys[r] & 0xFFFFFFFFull);
    const uint64_t deg = 0xFFFFFFFFull - (keys[r] >> 32);
    const bool last_heavy = deg >= P && (r + 1 == n || 0xFFFFFFFFull - (keys[r + 1] >> 32) < P);
    if (last_heavy) *heavy = (uint32_t)(r + 1);
}

__global__ void k_claim(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                        const int32_t* __restrict__ order, uint32_t r0, const int32_t* __restrict__ v2p,
                        int32_t* __restrict__ claim) {
    const int32_t rank = (int32_t)(r0 + blockIdx.x);
    const int32_t u = order[rank];
    for (uint64_t k = off[u] + threadIdx.x; k < off[u + 1]; k += blockDim.x) {
        const int32_t v = adj[k];
        if (v2p[v] < 0) atomicMin(&claim[v], rank);
    }
}

__device__ __forceinline__ uint64_t gcd64(uint64_t a, uint64_t b) {
    while (b) {
        const uint64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

__global__ void __launch_bounds__(kThreads) k_assign(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                                                     const int32_t* __restrict__ order, uint32_t r0, uint32_t r1,
                                                     uint32_t P, uint64_t key, const int32_t* __restrict__ claim,
                                                     int32_t* __restrict__ v2p) {
    extern __shared__ long long quota[];  // P + 1 entries: counts, then run starts
    using Reduce = cub::BlockReduce<long long, kThreads>;
    using Scan = cub::BlockScan<long long, kThreads>;
    __shared__ union {
        typename Reduce::TempStorage red;
        typename Scan::TempStorage scan;
    } tmp;
    __shared__ long long s_total, s_base;
    __shared__ unsigned long long s_a, s_b;
    const int32_t rank = (int32_t)(r0 + blockIdx.x);
    const int32_t u = order[rank];
    const uint64_t b = off[u], e = off[u + 1];
    const long long deg = (long long)(e - b);
    for (uint32_t k = threadIdx.x; k <= P; k += blockDim.x) quota[k] = 0;
    __syncthreads();
    // pass 1: neighbours placed before this wave, per partition; claimed count F
    long long mine = 0;
    for (uint64_t k = b + threadIdx.x; k < e; k += blockDim.x) {
        const int32_t v = adj[k];
        const int32_t c = claim[v];
        if (c == rank) ++mine;
        else if ((c < (int32_t)r0 || c >= (int32_t)r1) && v2p[v] >= 0) atomicAdd((unsigned long long*)&quota[v2p[v]], 1ull);
    }
    const long long F = Reduce(tmp.red).Sum(mine);
    if (threadIdx.x == 0) s_total = F;
    __syncthreads();
    if (s_total == 0) return;
    // quotas max(0, deg/P - count_i) and their sum
    const long long ulb = deg / (long long)P;
    long long part = 0;
    for (uint32_t k = threadIdx.x; k < P; k += blockDim.x) {
        const long long q = ulb - quota[k];
        quota[k] = q > 0 ? q : 0;
        part += quota[k];
    }
    __syncthreads();
    const long long psum = Reduce(tmp.red).Sum(part);
    if (threadIdx.x == 0) s_base = psum;
    __syncthreads();
    const long long sum = s_base, Ft = s_total;
    // run lengths p_i * F / sum, then run starts (exclusive prefix over P entries)
    const uint32_t per = (P + kThreads - 1) / kThreads;
    const uint32_t k0 = threadIdx.x * per, k1 = min(P, k0 + per);
    long long local = 0;
    for (uint32_t k = k0; k < k1; ++k) {
        const long long len = sum > 0 ? quota[k] * Ft / sum : 0;
        quota[k] = len;
        local += len;
    }
    long long start = 0;
    __syncthreads();
    Scan(tmp.scan).ExclusiveSum(local, start);
    for (uint32_t k = k0; k < k1; ++k) {
        const long long len = quota[k];
        quota[k] = start;
        start += len;
    }
    if (threadIdx.x == kThreads - 1) quota[P] = start;  // positions below this are placed by quota
    if (threadIdx.x == 0) {
        // seeded affine permutation k -> (a k + c) mod F with gcd(a, F) = 1
        const uint64_t h = pc_draw(key, 2 * (uint64_t)u);
        uint64_t a = (h % (uint64_t)Ft) | 1ull;
        while (gcd64(a, (uint64_t)Ft) != 1) a += 1;
        s_a = a % (uint64_t)Ft;
        s_b = pc_draw(key, 2 * (uint64_t)u + 1) % (uint64_t)Ft;
        s_base = 0;
    }
    __syncthreads();
    const long long placed = quota[P];
    const unsigned long long A = s_a ? s_a : 1ull, B = s_b;
    // pass 2: the k-th claimed neighbour in row order takes position perm(k)
    for (uint64_t k0r = b; k0r < e; k0r += blockDim.x) {
        const uint64_t k = k0r + threadIdx.x;
        int32_t v = -1;
        long long flag = 0;
        if (k < e) {
            v = adj[k];
            flag = claim[v] == rank ? 1 : 0;
        }
        long long pos = 0, chunk = 0;
        Scan(tmp.scan).ExclusiveSum(flag, pos, chunk);
        if (flag) {
            const long long idx = s_base + pos;
            const long long q = (long long)(((unsigned __int128)A * (unsigned long long)idx + B) % (unsigned long long)Ft);
            int32_t p;
            if (q < placed) {
                uint32_t lo = 0, hi = P;  // last run start <= q
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (quota[mid] <= q) lo = mid; else hi = mid;
                }
                p = (int32_t)lo;
            } else {
                p = (int32_t)(pc_draw(key ^ 0x5bd1e995ull, (uint64_t)v) % P);
            }
            v2p[v] = p;
        }
        __syncthreads();
        if (threadIdx.x == 0) s_base += chunk;
        __syncthreads();
    }
}

__global__ void k_place_rest(int32_t* __restrict__ v2p, uint64_t n, uint32_t P, uint64_t key) {
    const uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (v < n && v2p[v] < 0) v2p[v] = (int32_t)(pc_draw(key ^ 0x5bd1e995ull, v) % P);
}

}  // namespace part
}  // namespace pc

using namespace pc;
using namespace pc::part;

extern "C" {

pc_status pc_greedy_partition(pc_graph* g, int32_t P, uint64_t seed, int32_t* v2p_host) {
    clear_error();
    if (!g || !v2p_host) return fail(PC_ERR_INVALID_INPUT, "null argument");
    if (P < 1 || P > kMaxParts) return fail(PC_ERR_INVALID_INPUT, "partition count must be in [1, 16384]");
    PC_TRY(use_device(g));
    const uint64_t n = g->n;
    if (n == 0) return PC_OK;
    if (n >= 0x7F7F7F7Full) return fail(PC_ERR_UNSUPPORTED, "too many vertices for the claim words");
    cudaStream_t s = g->stream;
    const uint64_t key = pc_graph_key(seed, PC_GEN_PARTITION);
    DevBuf keys, order, v2p, claim, misc, tmpb;
    PC_TRY(keys.alloc(n * 16, "degree keys"));
    PC_TRY(order.alloc(n * 4, "order"));
    PC_TRY(v2p.alloc(n * 4, "vertex2partition"));
    PC_TRY(claim.alloc(n * 4, "claims"));
    PC_TRY(misc.alloc(16, "heavy count"));
    uint64_t* ka = keys.as<uint64_t>();
    cub::DoubleBuffer<uint64_t> db(ka, ka + n);
    size_t tb = 0;
    PC_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, db, (int64_t)n, 0, 64, s));
    PC_TRY(tmpb.alloc(std::max<size_t>(tb, 256), "sort scratch"));
    const unsigned nb = (unsigned)ceil_div(n, 256);
    k_degree_order_keys<<<nb, 256, 0, s>>>(g->off.as<uint64_t>(), n, ka);
    PC_LAUNCHED();
    PC_CUDA(cub::DeviceRadixSort::SortKeys(tmpb.p, tb, db, (int64_t)n, 0, 64, s));
    count_launch();
    PC_CUDA(cudaMemsetAsync(misc.p, 0, 16, s));
    k_order<<<nb, 256, 0, s>>>(db.Current(), n, (uint32_t)P, order.as<int32_t>(), misc.as<uint32_t>());
    PC_LAUNCHED();
    PC_CUDA(cudaMemsetAsync(v2p.p, 0xff, n * 4, s));   // -1: unplaced
    PC_CUDA(cudaMemsetAsync(claim.p, 0x7f, n * 4, s)); // above every rank (n < 2^31)
    uint32_t heavy = 0;
    PC_CUDA(cudaMemcpyAsync(&heavy, misc.p, 4, cudaMemcpyDeviceToHost, s));
    PC_CUDA(cudaStreamSynchronize(s));
    const size_t smem = (size_t)(P + 1) * sizeof(long long);
    PC_CUDA(cudaFuncSetAttribute(k_assign, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    for (uint32_t r0 = 0; r0 < heavy; r0 += kWave) {
        const uint32_t r1 = std::min<uint32_t>(heavy, r0 + kWave);
        k_claim<<<r1 - r0, kThreads, 0, s>>>(g->off.as<uint64_t>(), g->adj.as<int32_t>(), order.as<int32_t>(), r0,
                                              v2p.as<int32_t>(), claim.as<int32_t>());
        PC_LAUNCHED();
        k_assign<<<r1 - r0, kThreads, smem, s>>>(g->off.as<uint64_t>(), g->adj.as<int32_t>(), order.as<int32_t>(), r0,
                                                 r1, (uint32_t)P, key, claim.as<int32_t>(), v2p.as<int32_t>());
        PC_LAUNCHED();
    }
    k_place_rest<<<nb, 256, 0, s>>>(v2p.as<int32_t>(), n, (uint32_t)P, key);
    PC_LAUNCHED();
    PC_CUDA(cudaMemcpyAsync(v2p_host, v2p.p, n * 4, cudaMemcpyDeviceToHost, s));
    PC_CUDA(cudaStreamSynchronize(s));
    return PC_OK;
}

}  // extern "C"
