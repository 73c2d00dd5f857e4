// Multi-way neighbourhood queries on the intersection core (sm_100a):
// friend-triangle counts around a root and square (4-cycle) counting.
//
// Friend triangles (Partitioned_Graph::solve_friend_triangle_merge /
// _galloping, src/Graph.cpp:1222-1264; Graph:: forms :309-340): for the
// positions j < k of `nodes` whose vertex is not the root, the sum of
// |N(root) & N(nodes[j]) & N(nodes[k])| (summed over partitions, which
// partition each neighbour list).  With c_w = the number of such positions
// whose vertex is adjacent to w, the sum equals sum over w in N(root) of
// c_w (c_w - 1) / 2, so the GPU never enumerates the pairs: one warp per
// position intersects N(root) with N(nodes[j]) and counts hits per position
// of N(root); a reduction then sums the binomials.
//
// Squares (Partitioned_Graph::solve_square_counting, src/Graph.cpp:1291-1324):
// the reference lists the work items (v, w) for every u, v, w with w < v < u
// and v, w in N(u), and sums |N(v) & N(w) & [0, w)| over partitions, i.e.
// over the whole lists.  Here one warp per vertex u walks v over N+(u) =
// N(u) & [0, u); N+(v) goes into a warp-private hash (binary search when it
// is larger than the hash), and the lanes take the w in N+(u) below v and
// count the ids of N+(w) (all below w) that are in N+(v): x < w with x in
// N(v) is exactly x in N+(v).  The ordering conditions use the caller's ids,
// so after reorder() on a non-contiguous partition the count runs on a copy
// of the CSR relabelled to those ids.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <vector>

#include "pc_internal.cuh"
#include "tc_kernels.cuh"

namespace pc {
namespace qry {

constexpr int kWarps = 8;  // warps per CTA

__device__ __forceinline__ bool contains(const int32_t* __restrict__ p, uint32_t n, int32_t x, uint32_t* pos) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (p[mid] < x) lo = mid + 1; else hi = mid;
    }
    *pos = lo;
    return lo < n && p[lo] == x;
}

// cw[p] += 1 for every position p of N(root) whose id is adjacent to nodes[j].
__global__ void __launch_bounds__(kWarps * 32) k_friend_hits(const uint64_t* __restrict__ off,
                                                             const int32_t* __restrict__ adj, int32_t root,
                                                             const int32_t* __restrict__ nodes, uint64_t nn,
                                                             uint32_t* __restrict__ cw) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const int32_t* R = adj + off[root];
    const uint32_t dr = (uint32_t)(off[root + 1] - off[root]);
    for (uint64_t j = warp; j < nn; j += nwarps) {
        const int32_t x = nodes[j];
        if (x == root) continue;
        const int32_t* X = adj + off[x];
        const uint32_t dx = (uint32_t)(off[x + 1] - off[x]);
        uint32_t p;
        if (dx <= dr) {
            for (uint32_t i = lane; i < dx; i += 32)
                if (contains(R, dr, X[i], &p)) atomicAdd(&cw[p], 1u);
        } else {
            for (uint32_t i = lane; i < dr; i += 32)
                if (contains(X, dx, R[i], &p)) atomicAdd(&cw[i], 1u);
        }
    }
}

__global__ void k_binomial_sum(const uint32_t* __restrict__ cw, uint32_t n, unsigned long long* __restrict__ total) {
    unsigned long long s = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long c = cw[i];
        s += c * (c - (c ? 1 : 0)) / 2;
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(total, s);
}

// One warp per vertex u; see the file comment.
__global__ void __launch_bounds__(kWarps * 32) k_squares(const uint64_t* __restrict__ off,
                                                         const int32_t* __restrict__ adj,
                                                         const uint32_t* __restrict__ dplus, uint64_t n,
                                                         uint32_t* __restrict__ next_u,
                                                         unsigned long long* __restrict__ total) {
    __shared__ int32_t table[kWarps][tc::kHashSlots];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t* T = table[w];
    for (int s = lane; s < tc::kHashSlots; s += 32) T[s] = -1;
    __syncwarp();
    unsigned long long cnt = 0;
    for (;;) {
        uint32_t u = 0;
        if (lane == 0) u = atomicAdd(next_u, 1u);
        u = __shfl_sync(0xffffffffu, u, 0);
        if (u >= n) break;
        const int32_t* U = adj + off[u];
        const uint32_t du = dplus[u];
        for (uint32_t k = 1; k < du; ++k) {  // v = U[k]; w ranges over U[0..k)
            const int32_t v = U[k];
            const int32_t* V = adj + off[v];
            const uint32_t dv = dplus[v];
            const bool hashed = dv <= (uint32_t)tc::kHashCap;
            if (hashed) {
                for (uint32_t i = lane; i < dv; i += 32) {
                    const int32_t a = V[i];
                    uint32_t s = tc::hash_slot(a);
                    while (atomicCAS(&T[s], -1, a) != -1) s = (s + 1) & (tc::kHashSlots - 1);
                }
                __syncwarp();
            }
            for (uint32_t i = lane; i < k; i += 32) {
                const int32_t wv = U[i];
                const int32_t* Wr = adj + off[wv];
                const uint32_t dw = dplus[wv];
                for (uint32_t t = 0; t < dw; ++t) {
                    const int32_t x = Wr[t];
                    if (hashed) {
                        uint32_t s = tc::hash_slot(x);
                        int32_t key;
                        while ((key = T[s]) != -1) {
                            if (key == x) { ++cnt; break; }
                            s = (s + 1) & (tc::kHashSlots - 1);
                        }
                    } else {
                        uint32_t p;
                        if (contains(V, dv, x, &p)) ++cnt;
                    }
                }
            }
            if (hashed) {
                __syncwarp();
                for (int s = lane; s < tc::kHashSlots; s += 32) T[s] = -1;
                __syncwarp();
            }
        }
    }
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0 && cnt) atomicAdd(total, cnt);
}

// Keys old2new[u] * 2^B + old2new[v] of every CSR entry (warp per row).
__global__ void k_relabel_entry_keys(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj, uint64_t n,
                                     const int32_t* __restrict__ o2n, uint32_t B, uint64_t* __restrict__ keys) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t u = warp; u < n; u += nwarps) {
        const uint64_t nu = (uint64_t)o2n[u] << B;
        for (uint64_t k = off[u] + lane; k < off[u + 1]; k += 32) keys[k] = nu | (uint64_t)o2n[adj[k]];
    }
}

__global__ void k_keys_to_csr(const uint64_t* __restrict__ keys, uint64_t m, uint64_t n, uint32_t B,
                              uint64_t* __restrict__ off, int32_t* __restrict__ adj) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t mask = (1ull << B) - 1;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= m; i += stride) {
        const uint64_t row = i < m ? keys[i] >> B : n;
        const int64_t prev = i == 0 ? -1 : (int64_t)(keys[i - 1] >> B);
        for (int64_t r = prev + 1; r <= (int64_t)row; ++r) off[r] = i;
        if (i < m) adj[i] = (int32_t)(keys[i] & mask);
    }
}

__global__ void k_prefix_len(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj, uint64_t n,
                             uint32_t* __restrict__ dplus) {
    const uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (u >= n) return;
    uint64_t lo = off[u], hi = off[u + 1];
    const uint64_t b = lo;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (adj[mid] < (int32_t)u) lo = mid + 1; else hi = mid;
    }
    dplus[u] = (uint32_t)(lo - b);
}

}  // namespace qry
}  // namespace pc

using namespace pc;
using namespace pc::qry;

extern "C" {

pc_status pc_friend_triangle(pc_pgraph* pg, int32_t root, const int32_t* nodes, uint64_t nn, uint64_t* out) {
    clear_error();
    if (!pg || !out || (nn && !nodes)) return fail(PC_ERR_INVALID_INPUT, "null argument");
    const uint64_t n = pg->g->n;
    if (root < 0 || (uint64_t)root >= n) return fail(PC_ERR_INVALID_INPUT, "root vertex out of range");
    for (uint64_t i = 0; i < nn; ++i)
        if (nodes[i] < 0 || (uint64_t)nodes[i] >= n) return fail(PC_ERR_INVALID_INPUT, "query vertex out of range");
    *out = 0;
    if (nn < 2) return PC_OK;
    PC_TRY(use_device(pg->g));
    cudaStream_t s = pg->g->stream;
    const int32_t iroot = to_internal_id(pg, root);
    uint64_t dr = 0;
    {
        uint64_t o[2];
        PC_CUDA(cudaMemcpyAsync(o, pg->off + iroot, 16, cudaMemcpyDeviceToHost, s));
        PC_CUDA(cudaStreamSynchronize(s));
        dr = o[1] - o[0];
    }
    PC_TRY(scratch_reserve(pg, nn * 4 + dr * 4 + 1024));
    int32_t* d_nodes = nullptr;
    PC_TRY(upload(pg, nodes, nn, &d_nodes));
    PC_TRY(map_ids_to_internal(pg, d_nodes, nn));
    uint32_t* cw = pg->scratch.take<uint32_t>(std::max<uint64_t>(dr, 1));
    unsigned long long* d_total = pg->scratch.take<unsigned long long>(1);
    PC_CUDA(cudaMemsetAsync(cw, 0, std::max<uint64_t>(dr, 1) * 4, s));
    PC_CUDA(cudaMemsetAsync(d_total, 0, 8, s));
    const int sms = sm_count(pg->g->device);
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sms * 8, ceil_div(nn, kWarps)));
    k_friend_hits<<<grid, kWarps * 32, 0, s>>>(pg->off, pg->adj, iroot, d_nodes, nn, cw);
    PC_LAUNCHED();
    if (dr) {
        k_binomial_sum<<<(unsigned)std::min<uint64_t>((uint64_t)sms * 4, ceil_div(dr, 256)), 256, 0, s>>>(
            cw, (uint32_t)dr, d_total);
        PC_LAUNCHED();
    }
    unsigned long long h = 0;
    PC_CUDA(cudaMemcpyAsync(&h, d_total, 8, cudaMemcpyDeviceToHost, s));
    PC_TRY(sync(pg));
    *out = h;
    return PC_OK;
}

pc_status pc_square_count(pc_pgraph* pg, uint64_t* out) {
    clear_error();
    if (!pg || !out) return fail(PC_ERR_INVALID_INPUT, "null argument");
    PC_TRY(use_device(pg->g));
    cudaStream_t s = pg->g->stream;
    const uint64_t n = pg->g->n, m = pg->g->m;
    const int sms = sm_count(pg->g->device);
    *out = 0;
    if (n == 0 || m == 0) return PC_OK;
    const uint64_t* off = pg->off;
    const int32_t* adj = pg->adj;
    DevBuf roff, radj, keys, dp;
    if (!api_is_internal(pg)) {
        // the caller's id order: relabel the CSR by old2new and sort it
        uint32_t B = 1;
        while ((1ull << B) <= n) ++B;
        PC_TRY(keys.alloc(m * 16, "relabel keys"));
        PC_TRY(roff.alloc((n + 1) * 8, "relabelled offsets"));
        PC_TRY(radj.alloc((m + 64) * 4, "relabelled ids"));
        uint64_t* ka = keys.as<uint64_t>();
        cub::DoubleBuffer<uint64_t> db(ka, ka + m);
        size_t tb = 0;
        PC_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, db, (int64_t)m, 0, (int)(2 * B), s));
        DevBuf tmp;
        PC_TRY(tmp.alloc(std::max<size_t>(tb, 256), "sort scratch"));
        k_relabel_entry_keys<<<sms * 8, 256, 0, s>>>(off, adj, n, pg->old2new.as<int32_t>(), B, ka);
        PC_LAUNCHED();
        PC_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, tb, db, (int64_t)m, 0, (int)(2 * B), s));
        count_launch();
        k_keys_to_csr<<<(unsigned)std::min<uint64_t>((uint64_t)sms * 16, ceil_div(m + 1, 256)), 256, 0, s>>>(
            db.Current(), m, n, B, roff.as<uint64_t>(), radj.as<int32_t>());
        PC_LAUNCHED();
        PC_CUDA(cudaStreamSynchronize(s));  // tmp and keys are released on return
        off = roff.as<uint64_t>();
        adj = radj.as<int32_t>();
    }
    PC_TRY(dp.alloc(n * 4 + 64, "prefix lengths"));
    uint32_t* d_dplus = dp.as<uint32_t>();
    uint32_t* d_next = reinterpret_cast<uint32_t*>(dp.as<char>() + ((n * 4 + 15) & ~(uint64_t)15));
    unsigned long long* d_total = reinterpret_cast<unsigned long long*>(d_next + 4);
    PC_CUDA(cudaMemsetAsync(d_next, 0, 32, s));
    k_prefix_len<<<(unsigned)ceil_div(n, 256), 256, 0, s>>>(off, adj, n, d_dplus);
    PC_LAUNCHED();
    k_squares<<<sms * 8, kWarps * 32, 0, s>>>(off, adj, d_dplus, n, d_next, d_total);
    PC_LAUNCHED();
    unsigned long long h = 0;
    PC_CUDA(cudaMemcpyAsync(&h, d_total, 8, cudaMemcpyDeviceToHost, s));
    PC_TRY(sync(pg));
    *out = h;
    return PC_OK;
}

}  // extern "C"
