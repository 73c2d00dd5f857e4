// LCC and all-edge Jaccard on top of the triangle-count kernels, Jaccard
// over a query list, and batched pair / k-set intersection counts (sm_100a).
//
// Per-edge counts c({u,v}) = |N(u) & N(v)| come from the triangle-count
// kernels in per-edge mode (tc_edge_triangles): every triangle adds 1 to its
// three edges.  An undirected edge {x, y}, y < x, is counted at its oriented
// slot: position k of y in row x (k < dplus[x]).  A finalisation pass reads,
// for every CSR entry, its own slot or its twin's and forms the Jaccard ratio
// exactly as the reference defines it (src/Graph.cpp:798-812).  LCC needs only
// per-vertex triangle counts (tc_vertex_triangles).
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>

#include "pc_internal.cuh"
#include "selector.cuh"

namespace pc {
namespace ix {

// lower_bound of x in sorted p[0..n)
__device__ __forceinline__ uint32_t lb(const int32_t* __restrict__ p, uint32_t n, int32_t x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (p[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Count of the undirected edge behind CSR entry (u, v) at position e.
__device__ __forceinline__ uint32_t edge_count(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                                               const uint32_t* __restrict__ dplus, const uint32_t* __restrict__ ecnt,
                                               uint64_t u, int32_t v, uint64_t e) {
    if ((uint64_t)v < u) return ecnt[e];
    const uint64_t rv = off[v];
    return ecnt[rv + lb(adj + rv, dplus[v], (int32_t)u)];
}

// Largest row r in [lo, hi] with off[r] <= j (off[lo] <= j < off[hi + 1]):
// the row that holds CSR entry j, empty rows skipped.
__device__ __forceinline__ uint64_t row_of(const uint64_t* __restrict__ off, uint64_t lo, uint64_t hi, uint64_t j) {
    while (lo < hi) {
        const uint64_t mid = (lo + hi + 1) >> 1;
        if (off[mid] <= j) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Jaccard per CSR entry (fp32 output of the fp64 formula).  The work is split
// by entries, not rows: each warp takes kJacChunk consecutive entries, finds
// the rows at both ends of its chunk, and each lane finds the row of its own
// entries inside that span, so a hub row is spread over many warps instead
// of serialising one.
constexpr uint64_t kJacChunk = 256;
__global__ void k_jaccard_entries(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                                  const uint32_t* __restrict__ dplus, const uint32_t* __restrict__ ecnt, uint64_t n,
                                  uint64_t m, float* __restrict__ jac) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t c0 = warp * kJacChunk; c0 < m; c0 += nwarps * kJacChunk) {
        const uint64_t c1 = min(c0 + kJacChunk, m);
        uint64_t r = 0;
        if (lane < 2) r = row_of(off, 0, n - 1, lane == 0 ? c0 : c1 - 1);
        const uint64_t r0 = __shfl_sync(0xffffffffu, r, 0), r1 = __shfl_sync(0xffffffffu, r, 1);
        for (uint64_t j = c0 + lane; j < c1; j += 32) {
            const uint64_t u = row_of(off, r0, r1, j);
            const int32_t v = adj[j];
            const uint32_t c = edge_count(off, adj, dplus, ecnt, u, v, j);
            const uint64_t du = off[u + 1] - off[u], dv = off[v + 1] - off[v];
            // src/Graph.cpp:808-809: c / (deg_u + deg_v - c), in double
            jac[j] = (float)((double)c / ((double)(du + dv) - (double)c));
        }
    }
}

// |N(a) & N(b)| for each pair: lanes take ids of the shorter list and look
// them up in the longer one by binary search (galloping probing).
__global__ void k_pair_counts(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                              const int32_t* __restrict__ pairs, uint64_t nq, unsigned long long* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t q = warp; q < nq; q += nwarps) {
        int32_t a = pairs[2 * q], b = pairs[2 * q + 1];
        uint64_t ra = off[a], la = off[a + 1] - ra, rb = off[b], lb_ = off[b + 1] - rb;
        if (la > lb_) { uint64_t t = ra; ra = rb; rb = t; t = la; la = lb_; lb_ = t; }
        unsigned long long c = 0;
        for (uint64_t i = lane; i < la; i += 32) {
            const int32_t x = adj[ra + i];
            const uint32_t p = lb(adj + rb, (uint32_t)lb_, x);
            c += (p < lb_ && adj[rb + p] == x) ? 1 : 0;
        }
        for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) out[q] = c;
    }
}

// |AND_j N(s_j)| for each k-set: ids of the shortest list looked up in all others.
__global__ void k_set_counts(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                             const int32_t* __restrict__ ids, const uint64_t* __restrict__ soff, uint64_t nq,
                             unsigned long long* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t q = warp; q < nq; q += nwarps) {
        const uint64_t s0 = soff[q], s1 = soff[q + 1];
        // shortest list
        uint64_t best = s0, bestlen = ~0ull;
        for (uint64_t t = s0; t < s1; ++t) {
            const int32_t v = ids[t];
            const uint64_t l = off[v + 1] - off[v];
            if (l < bestlen) { bestlen = l; best = t; }
        }
        const int32_t sv = ids[best];
        const uint64_t rs = off[sv];
        unsigned long long c = 0;
        for (uint64_t i = lane; i < bestlen; i += 32) {
            const int32_t x = adj[rs + i];
            bool all = true;
            for (uint64_t t = s0; t < s1 && all; ++t) {
                if (t == best) continue;
                const int32_t v = ids[t];
                const uint64_t rv = off[v], lv = off[v + 1] - rv;
                const uint32_t p = lb(adj + rv, (uint32_t)lv, x);
                all = p < lv && adj[rv + p] == x;
            }
            c += all ? 1 : 0;
        }
        for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) out[q] = c;
    }
}

__global__ void k_jaccard_pairs(const uint64_t* __restrict__ off, const int32_t* __restrict__ q, int32_t nq,
                                const unsigned long long* __restrict__ c, double* __restrict__ out) {
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (t >= (uint64_t)nq * nq) return;
    const int32_t i = (int32_t)(t / nq), j = (int32_t)(t % nq);
    const uint64_t du = off[q[i] + 1] - off[q[i]], dv = off[q[j] + 1] - off[q[j]];
    const double cc = (double)c[t];
    out[t] = cc / ((double)(du + dv) - cc);  // src/Graph.cpp:808-809
}

__global__ void k_make_pairs(const int32_t* __restrict__ q, int32_t nq, int32_t* __restrict__ pairs) {
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (t >= (uint64_t)nq * nq) return;
    pairs[2 * t] = q[t / nq];
    pairs[2 * t + 1] = q[t % nq];
}

}  // namespace ix

using namespace ix;

}  // namespace pc

using namespace pc;

extern "C" {

// LCC from per-vertex triangle counts: sum over v in N(u) of |N(u) & N(v)|
// counts every triangle at u twice, so the reference's numerator
// (src/Graph.cpp:2230-2261, 814-840) is exactly 2 t(u); the same single
// IEEE division follows, NaN at degree 1 as in the reference.
__global__ void k_lcc_from_triangles(const uint64_t* __restrict__ off, const unsigned long long* __restrict__ tri,
                                     uint64_t n, double* __restrict__ lcc) {
    const uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (u >= n) return;
    const uint64_t du = off[u + 1] - off[u];
    lcc[u] = du < 1 ? 0.0 : (double)(2 * tri[u]) / (double)(du * (du - 1));
}

pc_status pc_lcc(pc_pgraph* pg, int32_t method, double* out) {
    clear_error();
    if (!pg || !out) return fail(PC_ERR_INVALID_INPUT, "null argument");
    if (method != PC_METHOD_MERGE && method != PC_METHOD_GALLOPING) return fail(PC_ERR_INVALID_INPUT, "unknown method");
    PC_TRY(use_device(pg->g));
    const uint64_t n = pg->g->n;
    if (n == 0) return PC_OK;
    cudaStream_t s = pg->g->stream;
    // per-vertex triangle counts with the triangle-count plan (its variants,
    // the learned or heuristic choice per unit) in per-vertex mode
    DevBuf tri;
    PC_TRY(tri.alloc(n * 8, "triangles per vertex"));
    PC_CUDA(cudaMemsetAsync(tri.p, 0, n * 8, s));
    uint64_t T = 0;
    PC_TRY(tc_vertex_triangles(pg, PC_VARIANT_AUTO, tri.as<unsigned long long>(), &T));
    PC_TRY(scratch_reserve(pg, n * 16 + 1024));
    double* lcc = pg->scratch.take<double>(n);
    double* lcc_api = pg->scratch.take<double>(n);
    k_lcc_from_triangles<<<(unsigned)ceil_div(n, 256), 256, 0, s>>>(pg->off, tri.as<unsigned long long>(), n, lcc);
    PC_LAUNCHED();
    PC_TRY(gather_to_api_f64(pg, lcc, lcc_api));
    PC_CUDA(cudaMemcpyAsync(out, lcc_api, n * 8, cudaMemcpyDeviceToHost, s));
    return sync(pg);
}

pc_status pc_jaccard_edges(pc_pgraph* pg, float* out) {
    clear_error();
    if (!pg || !out) return fail(PC_ERR_INVALID_INPUT, "null argument");
    PC_TRY(use_device(pg->g));
    const uint64_t n = pg->g->n, m = pg->g->m;
    if (m == 0) return PC_OK;
    cudaStream_t s = pg->g->stream;
    // per-edge triangle counts with the triangle-count plan (its variants,
    // the learned or heuristic choice per unit) in per-edge mode
    DevBuf ecnt;
    PC_TRY(ecnt.alloc(m * 4, "triangles per edge"));
    PC_CUDA(cudaMemsetAsync(ecnt.p, 0, m * 4, s));
    uint64_t T = 0;
    PC_TRY(tc_edge_triangles(pg, PC_VARIANT_AUTO, ecnt.as<uint32_t>(), &T));
    PC_TRY(scratch_reserve(pg, m * 4 + 1024));
    float* jac = pg->scratch.take<float>(m);
    k_jaccard_entries<<<sm_count(pg->g->device) * 8, 256, 0, s>>>(pg->off, pg->adj, pg->dplus.as<uint32_t>(),
                                                                   ecnt.as<uint32_t>(), n, m, jac);
    PC_LAUNCHED();
    // entries are in the graph's own CSR order (internal ids are the graph's ids)
    PC_CUDA(cudaMemcpyAsync(out, jac, m * 4, cudaMemcpyDeviceToHost, s));
    return sync(pg);
}

pc_status pc_batch_count_pairs(pc_pgraph* pg, const int32_t* pairs, uint64_t nq, uint64_t* out) {
    clear_error();
    if (!pg || (nq && (!pairs || !out))) return fail(PC_ERR_INVALID_INPUT, "null argument");
    if (nq == 0) return PC_OK;
    const uint64_t n = pg->g->n;
    for (uint64_t i = 0; i < 2 * nq; ++i)
        if (pairs[i] < 0 || (uint64_t)pairs[i] >= n) return fail(PC_ERR_INVALID_INPUT, "query vertex out of range");
    PC_TRY(use_device(pg->g));
    cudaStream_t s = pg->g->stream;
    PC_TRY(scratch_reserve(pg, nq * 8 + nq * 8 + 512));
    int32_t* d_pairs = nullptr;
    PC_TRY(upload(pg, pairs, 2 * nq, &d_pairs));
    PC_TRY(map_ids_to_internal(pg, d_pairs, 2 * nq));
    unsigned long long* d_out = pg->scratch.take<unsigned long long>(nq);
    k_pair_counts<<<sm_count(pg->g->device) * 16, 256, 0, s>>>(pg->off, pg->adj, d_pairs, nq, d_out);
    PC_LAUNCHED();
    PC_CUDA(cudaMemcpyAsync(out, d_out, nq * 8, cudaMemcpyDeviceToHost, s));
    return sync(pg);
}

pc_status pc_batch_count_sets(pc_pgraph* pg, const int32_t* ids, const uint64_t* offsets, uint64_t nq, uint64_t* out) {
    clear_error();
    if (!pg || (nq && (!ids || !offsets || !out))) return fail(PC_ERR_INVALID_INPUT, "null argument");
    if (nq == 0) return PC_OK;
    const uint64_t n = pg->g->n;
    if (offsets[0] != 0) return fail(PC_ERR_INVALID_INPUT, "offsets[0] must be 0");
    for (uint64_t i = 0; i < nq; ++i)
        if (offsets[i + 1] <= offsets[i]) return fail(PC_ERR_INVALID_INPUT, "every set needs at least one vertex");
    const uint64_t tot = offsets[nq];
    for (uint64_t i = 0; i < tot; ++i)
        if (ids[i] < 0 || (uint64_t)ids[i] >= n) return fail(PC_ERR_INVALID_INPUT, "query vertex out of range");
    PC_TRY(use_device(pg->g));
    cudaStream_t s = pg->g->stream;
    PC_TRY(scratch_reserve(pg, tot * 4 + (nq + 1) * 8 + nq * 8 + 512));
    int32_t* d_ids = nullptr;
    uint64_t* d_off = nullptr;
    PC_TRY(upload(pg, ids, tot, &d_ids));
    PC_TRY(upload(pg, offsets, nq + 1, &d_off));
    PC_TRY(map_ids_to_internal(pg, d_ids, tot));
    unsigned long long* d_out = pg->scratch.take<unsigned long long>(nq);
    k_set_counts<<<sm_count(pg->g->device) * 16, 256, 0, s>>>(pg->off, pg->adj, d_ids, d_off, nq, d_out);
    PC_LAUNCHED();
    PC_CUDA(cudaMemcpyAsync(out, d_out, nq * 8, cudaMemcpyDeviceToHost, s));
    return sync(pg);
}

pc_status pc_jaccard_queries(pc_pgraph* pg, const int32_t* queries, int32_t nq, double* out) {
    clear_error();
    if (!pg || nq < 0 || (nq && (!queries || !out))) return fail(PC_ERR_INVALID_INPUT, "bad argument");
    if (nq == 0) return PC_OK;
    const uint64_t n = pg->g->n;
    for (int32_t i = 0; i < nq; ++i)
        if (queries[i] < 0 || (uint64_t)queries[i] >= n) return fail(PC_ERR_INVALID_INPUT, "query vertex out of range");
    PC_TRY(use_device(pg->g));
    cudaStream_t s = pg->g->stream;
    const uint64_t np = (uint64_t)nq * nq;
    PC_TRY(scratch_reserve(pg, nq * 4 + np * 8 + np * 8 + np * 8 + 512));
    int32_t* d_q = nullptr;
    PC_TRY(upload(pg, queries, (size_t)nq, &d_q));
    PC_TRY(map_ids_to_internal(pg, d_q, nq));
    int32_t* d_pairs = pg->scratch.take<int32_t>(2 * np);
    unsigned long long* d_c = pg->scratch.take<unsigned long long>(np);
    double* d_out = pg->scratch.take<double>(np);
    k_make_pairs<<<(unsigned)ceil_div(np, 256), 256, 0, s>>>(d_q, nq, d_pairs);
    PC_LAUNCHED();
    k_pair_counts<<<sm_count(pg->g->device) * 16, 256, 0, s>>>(pg->off, pg->adj, d_pairs, np, d_c);
    PC_LAUNCHED();
    k_jaccard_pairs<<<(unsigned)ceil_div(np, 256), 256, 0, s>>>(pg->off, d_q, nq, d_c, d_out);
    PC_LAUNCHED();
    PC_CUDA(cudaMemcpyAsync(out, d_out, np * 8, cudaMemcpyDeviceToHost, s));
    return sync(pg);
}

}  // extern "C"
