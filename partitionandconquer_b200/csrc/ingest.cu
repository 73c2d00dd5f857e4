// GPU ingest: a raw edge stream becomes, on the device, the symmetric CSR
// with sorted, duplicate-free rows and no self-loops that the reference's
// loaders produce; optionally the vertices are relabelled by descending
// degree (ties by ascending id).
//
// Reference: the adjacency build of the text loader (src/Graph.cpp:59-85:
// both directions of every edge, self-loops dropped, rows sorted and
// deduplicated) and the preprocess tool (src/preprocess.cpp:5-45), which
// writes the resulting csr_vlist.bin / csr_elist.bin.  The host builders
// (host/host_csr.cpp: build_symmetric_csr, relabel_by_degree, gen_rmat,
// gen_er, add_weights) compute the same arrays on the CPU.
//
// Method.  With B = bits(n), every edge (u, v), u != v, gives the two keys
// u * 2^B + v and v * 2^B + u; a self-loop gives the key n * 2^B.  One radix
// sort over 2B bits orders the keys row-major, a unique pass drops repeated
// edges, and one pass over the sorted keys writes csr_elist and csr_vlist
// (a row starts where the row part of the key changes).  The degree relabel
// sorts (2^32 - 1 - deg) * 2^32 + id, scatters old -> new, rewrites every key
// and sorts once more.  Nothing here is data-dependent control on the host:
// the only host reads are the unique count and the last key.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>

#include "pc_internal.cuh"
#include "synth_rng.h"

namespace pc {
namespace ingest {

__device__ __forceinline__ uint64_t edge_key(uint32_t u, uint32_t v, uint32_t B) {
    return ((uint64_t)u << B) | v;
}

// Keys of a caller edge stream; ids outside [0, n) raise *bad.
__global__ void k_keys_from_edges(const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst, uint64_t ne,
                                  uint64_t n, uint32_t B, uint64_t* __restrict__ keys, uint32_t* __restrict__ bad) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t self = (uint64_t)n << B;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < ne; k += stride) {
        const uint32_t u = src[k], v = dst[k];
        if (u >= n || v >= n) {
            atomicOr(bad, 1u);
            keys[2 * k] = keys[2 * k + 1] = self;
            continue;
        }
        keys[2 * k] = u == v ? self : edge_key(u, v, B);
        keys[2 * k + 1] = u == v ? self : edge_key(v, u, B);
    }
}

// Keys of the seeded generators (the host generators' edge streams).
template <int kKind>
__global__ void k_keys_synth(uint64_t genkey, uint32_t scale, uint64_t ne, uint32_t B, uint64_t* __restrict__ keys) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t self = (1ull << scale) << B;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < ne; k += stride) {
        uint32_t u, v;
        if (kKind == PC_GEN_RMAT) pc_rmat_edge(genkey, k, scale, &u, &v);
        else pc_er_edge(genkey, k, scale, &u, &v);
        keys[2 * k] = u == v ? self : edge_key(u, v, B);
        keys[2 * k + 1] = u == v ? self : edge_key(v, u, B);
    }
}

// csr_elist[i] = column of key i; csr_vlist[r] = first i whose row is >= r.
__global__ void k_csr_from_keys(const uint64_t* __restrict__ keys, uint64_t m, uint64_t n, uint32_t B,
                                uint64_t* __restrict__ off, int32_t* __restrict__ adj) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t mask = (1ull << B) - 1;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= m; i += stride) {
        const uint64_t row = i < m ? keys[i] >> B : n;
        const int64_t prev = i == 0 ? -1 : (int64_t)(keys[i - 1] >> B);
        for (int64_t r = prev + 1; r <= (int64_t)row; ++r) off[r] = i;
        if (adj && i < m) adj[i] = (int32_t)(keys[i] & mask);
    }
}

// (2^32 - 1 - deg(u)) * 2^32 + u: ascending order = descending degree, ties by id.
__global__ void k_degree_keys(const uint64_t* __restrict__ off, uint64_t n, uint64_t* __restrict__ rk) {
    const uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (u >= n) return;
    rk[u] = ((0xFFFFFFFFull - (off[u + 1] - off[u])) << 32) | u;
}

__global__ void k_scatter_rank(const uint64_t* __restrict__ rk, uint64_t n, int32_t* __restrict__ old2new) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    old2new[rk[i] & 0xFFFFFFFFull] = (int32_t)i;
}

__global__ void k_relabel_keys(const uint64_t* __restrict__ in, uint64_t m, uint32_t B,
                               const int32_t* __restrict__ old2new, uint64_t* __restrict__ out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t mask = (1ull << B) - 1;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += stride) {
        const uint64_t k = in[i];
        out[i] = edge_key((uint32_t)old2new[k >> B], (uint32_t)old2new[k & mask], B);
    }
}

// Symmetric weights keyed on the unordered pair (host add_weights).
__global__ void k_weights(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj, uint64_t n,
                          uint64_t key, int32_t wmax, int32_t* __restrict__ w) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t u = warp; u < n; u += nwarps)
        for (uint64_t k = off[u] + lane; k < off[u + 1]; k += 32)
            w[k] = pc_edge_weight(key, (uint32_t)u, (uint32_t)adj[k], wmax);
}

static uint32_t bits_for(uint64_t n) {
    uint32_t b = 1;
    while ((1ull << b) <= n) ++b;
    return b;
}

// New handle with its own stream on the current device (no arrays yet).
static pc_status new_handle(uint64_t n, pc_graph** out) {
    pc_graph* g = new pc_graph();
    cudaError_t e = cudaGetDevice(&g->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        if (g->stream) cudaStreamDestroy(g->stream);
        delete g;
        return cuda_fail(e, "graph handle", __FILE__, __LINE__);
    }
    g->n = n;
    *out = g;
    return PC_OK;
}

static void drop_handle(pc_graph* g) {
    if (!g) return;
    if (g->stream) {
        cudaStreamSynchronize(g->stream);
        cudaStreamDestroy(g->stream);
    }
    delete g;
}

// Sorts 2*ne keys held in a[] (b[] is the same size), drops duplicates and
// self-loop keys, and writes the CSR into g; relabels when asked.
static pc_status keys_to_graph(pc_graph* g, DevBuf& a, DevBuf& b, uint64_t nkeys, uint32_t B, bool relabel,
                               int32_t* old2new_host) {
    cudaStream_t s = g->stream;
    const uint64_t n = g->n;
    const int sms = sm_count(g->device);
    uint64_t* ka = a.as<uint64_t>();
    uint64_t* kb = b.as<uint64_t>();
    const int end_bit = (int)(2 * B);
    DevBuf tmp, cnt;
    PC_TRY(cnt.alloc(16, "unique count"));
    size_t tb_sort = 0, tb_uniq = 0;
    cub::DoubleBuffer<uint64_t> db(ka, kb);
    PC_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb_sort, db, (int64_t)nkeys, 0, end_bit, s));
    PC_CUDA(cub::DeviceSelect::Unique(nullptr, tb_uniq, ka, kb, cnt.as<uint64_t>(), (int64_t)nkeys, s));
    PC_TRY(tmp.alloc(std::max<size_t>({tb_sort, tb_uniq, 256}), "sort scratch"));
    PC_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, tb_sort, db, (int64_t)nkeys, 0, end_bit, s));
    count_launch();
    uint64_t* sorted = db.Current();
    uint64_t* uniq = db.Alternate();
    PC_CUDA(cub::DeviceSelect::Unique(tmp.p, tb_uniq, sorted, uniq, cnt.as<uint64_t>(), (int64_t)nkeys, s));
    count_launch();
    uint64_t nu = 0;
    PC_CUDA(cudaMemcpyAsync(&nu, cnt.p, 8, cudaMemcpyDeviceToHost, s));
    PC_CUDA(cudaStreamSynchronize(s));
    uint64_t last = 0;
    if (nu) {
        PC_CUDA(cudaMemcpyAsync(&last, uniq + nu - 1, 8, cudaMemcpyDeviceToHost, s));
        PC_CUDA(cudaStreamSynchronize(s));
    }
    const uint64_t m = (nu && (last >> B) == n) ? nu - 1 : nu;  // the self-loop key sorts last
    g->m = m;
    PC_TRY(g->off.alloc((n + 1) * 8, "csr_vlist"));
    PC_TRY(g->adj.alloc((m + 64) * 4, "csr_elist"));
    PC_CUDA(cudaMemsetAsync(g->adj.as<int32_t>() + m, 0x7f, 64 * 4, s));
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sms * 16, ceil_div(m + 1, 256)));
    if (!relabel) {
        k_csr_from_keys<<<grid, 256, 0, s>>>(uniq, m, n, B, g->off.as<uint64_t>(), g->adj.as<int32_t>());
        PC_LAUNCHED();
        PC_CUDA(cudaStreamSynchronize(s));
        return PC_OK;
    }
    // offsets of the unrelabelled graph give the degrees
    k_csr_from_keys<<<grid, 256, 0, s>>>(uniq, m, n, B, g->off.as<uint64_t>(), nullptr);
    PC_LAUNCHED();
    DevBuf rk, o2n;
    PC_TRY(rk.alloc(std::max<uint64_t>(n, 1) * 16, "degree keys"));
    PC_TRY(o2n.alloc(std::max<uint64_t>(n, 1) * 4, "old2new"));
    uint64_t* rka = rk.as<uint64_t>();
    uint64_t* rkb = rka + n;
    k_degree_keys<<<(unsigned)ceil_div(std::max<uint64_t>(n, 1), 256), 256, 0, s>>>(g->off.as<uint64_t>(), n, rka);
    PC_LAUNCHED();
    cub::DoubleBuffer<uint64_t> rdb(rka, rkb);
    size_t tb_r = 0;
    PC_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb_r, rdb, (int64_t)n, 0, 64, s));
    if (tb_r > tmp.bytes) {  // nothing in flight uses tmp after the sync above
        PC_TRY(tmp.alloc(tb_r, "sort scratch"));
    }
    PC_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, tb_r, rdb, (int64_t)n, 0, 64, s));
    count_launch();
    k_scatter_rank<<<(unsigned)ceil_div(std::max<uint64_t>(n, 1), 256), 256, 0, s>>>(rdb.Current(), n,
                                                                                     o2n.as<int32_t>());
    PC_LAUNCHED();
    // rewrite the m edge keys into the other buffer and sort them again
    uint64_t* other = (uniq == ka) ? kb : ka;
    k_relabel_keys<<<grid, 256, 0, s>>>(uniq, m, B, o2n.as<int32_t>(), other);
    PC_LAUNCHED();
    cub::DoubleBuffer<uint64_t> edb(other, uniq);
    size_t tb_e = 0;
    PC_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb_e, edb, (int64_t)m, 0, end_bit, s));
    if (tb_e > tmp.bytes) {
        PC_CUDA(cudaStreamSynchronize(s));  // the degree sort may still use tmp
        PC_TRY(tmp.alloc(tb_e, "sort scratch"));
    }
    PC_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, tb_e, edb, (int64_t)m, 0, end_bit, s));
    count_launch();
    k_csr_from_keys<<<grid, 256, 0, s>>>(edb.Current(), m, n, B, g->off.as<uint64_t>(), g->adj.as<int32_t>());
    PC_LAUNCHED();
    if (old2new_host && n)
        PC_CUDA(cudaMemcpyAsync(old2new_host, o2n.p, n * 4, cudaMemcpyDeviceToHost, s));
    PC_CUDA(cudaStreamSynchronize(s));
    return PC_OK;
}

static pc_status check_n(uint64_t n) {
    if (n == 0) return fail(PC_ERR_INVALID_INPUT, "the graph needs at least one vertex");
    if (n >= (1ull << 31)) return fail(PC_ERR_INVALID_INPUT, "vertex count exceeds the int32 id range");
    if (pc_device_count() == 0) return fail(PC_ERR_NO_DEVICE, "no CUDA device is visible");
    return PC_OK;
}

template <int kKind>
static pc_status synth_graph(uint32_t scale, uint64_t ne, uint64_t seed, uint32_t flags, pc_graph** out) {
    if (!out) return fail(PC_ERR_INVALID_INPUT, "out is null");
    *out = nullptr;
    if (scale == 0 || scale > 30) return fail(PC_ERR_INVALID_INPUT, "scale must be in [1, 30]");
    const uint64_t n = 1ull << scale;
    PC_TRY(check_n(n));
    pc_graph* g = nullptr;
    PC_TRY(new_handle(n, &g));
    const uint32_t B = bits_for(n);
    DevBuf a, b;
    pc_status st = a.alloc(std::max<uint64_t>(2 * ne, 1) * 8, "edge keys");
    if (st == PC_OK) st = b.alloc(std::max<uint64_t>(2 * ne, 1) * 8, "edge keys");
    if (st == PC_OK) {
        const int sms = sm_count(g->device);
        const uint64_t key = pc_graph_key(seed, (uint64_t)kKind);
        k_keys_synth<kKind><<<sms * 16, 256, 0, g->stream>>>(key, scale, ne, B, a.as<uint64_t>());
        cudaError_t e = cudaGetLastError();
        count_launch();
        st = e == cudaSuccess ? keys_to_graph(g, a, b, 2 * ne, B, (flags & PC_INGEST_DEGREE_RELABEL) != 0, nullptr)
                              : cuda_fail(e, "kernel launch", __FILE__, __LINE__);
    }
    if (st != PC_OK) {
        const std::string msg = pc_last_error();
        drop_handle(g);
        return fail(st, msg);
    }
    *out = g;
    return PC_OK;
}

}  // namespace ingest
}  // namespace pc

using namespace pc;
using namespace pc::ingest;

extern "C" {

pc_status pc_graph_from_edges(const uint32_t* src, const uint32_t* dst, uint64_t nedges, uint64_t n, uint32_t flags,
                              int32_t* old2new, pc_graph** out) {
    clear_error();
    if (!out) return fail(PC_ERR_INVALID_INPUT, "out is null");
    *out = nullptr;
    if (nedges && (!src || !dst)) return fail(PC_ERR_INVALID_INPUT, "edge arrays are null");
    PC_TRY(check_n(n));
    pc_graph* g = nullptr;
    PC_TRY(new_handle(n, &g));
    const uint32_t B = bits_for(n);
    DevBuf a, b, raw;
    pc_status st = a.alloc(std::max<uint64_t>(2 * nedges, 1) * 8, "edge keys");
    if (st == PC_OK) st = b.alloc(std::max<uint64_t>(2 * nedges, 1) * 8, "edge keys");
    // the raw stream is staged in b (its first half holds src, then dst)
    if (st == PC_OK) st = raw.alloc(16, "input check");
    if (st == PC_OK) {
        cudaStream_t s = g->stream;
        uint32_t* d_src = b.as<uint32_t>();
        uint32_t* d_dst = d_src + nedges;
        cudaError_t e = cudaMemsetAsync(raw.p, 0, 16, s);
        if (e == cudaSuccess && nedges) e = cudaMemcpyAsync(d_src, src, nedges * 4, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && nedges) e = cudaMemcpyAsync(d_dst, dst, nedges * 4, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && nedges) {
            const int sms = sm_count(g->device);
            k_keys_from_edges<<<sms * 16, 256, 0, s>>>(d_src, d_dst, nedges, n, B, a.as<uint64_t>(), raw.as<uint32_t>());
            e = cudaGetLastError();
            count_launch();
        }
        uint32_t bad = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, raw.p, 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "edge upload", __FILE__, __LINE__);
        else if (bad) st = fail(PC_ERR_INVALID_INPUT, "an edge endpoint is outside [0, n)");
        else st = keys_to_graph(g, a, b, 2 * nedges, B, (flags & PC_INGEST_DEGREE_RELABEL) != 0, old2new);
    }
    if (st != PC_OK) {
        const std::string msg = pc_last_error();
        drop_handle(g);
        return fail(st, msg);
    }
    *out = g;
    return PC_OK;
}

pc_status pc_graph_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, uint32_t flags, pc_graph** out) {
    clear_error();
    return synth_graph<PC_GEN_RMAT>(scale, ((uint64_t)1 << scale) * edge_factor, seed, flags, out);
}

pc_status pc_graph_er(uint32_t scale, uint64_t nedges, uint64_t seed, uint32_t flags, pc_graph** out) {
    clear_error();
    return synth_graph<PC_GEN_ER>(scale, nedges, seed, flags, out);
}

pc_status pc_graph_add_weights(pc_graph* g, uint64_t seed, int32_t wmax) {
    clear_error();
    if (!g) return fail(PC_ERR_INVALID_INPUT, "null graph");
    if (wmax < 1 || wmax >= (1 << 30)) return fail(PC_ERR_INVALID_INPUT, "wmax must be in [1, 2^30)");
    if (g->live_views) return fail(PC_ERR_UNSUPPORTED, "weights cannot change while a partitioned view exists");
    PC_TRY(use_device(g));
    if (!g->weighted) PC_TRY(g->w.alloc(std::max<uint64_t>(g->m, 1) * 4, "csr_weight"));
    const int sms = sm_count(g->device);
    k_weights<<<sms * 8, 256, 0, g->stream>>>(g->off.as<uint64_t>(), g->adj.as<int32_t>(), g->n,
                                              pc_graph_key(seed, PC_GEN_WEIGHT), wmax, g->w.as<int32_t>());
    PC_LAUNCHED();
    PC_CUDA(cudaStreamSynchronize(g->stream));
    g->weighted = true;
    return PC_OK;
}

pc_status pc_graph_download(const pc_graph* g, uint64_t* vlist, int32_t* elist, int32_t* weights) {
    clear_error();
    if (!g) return fail(PC_ERR_INVALID_INPUT, "null graph");
    if (weights && !g->weighted) return fail(PC_ERR_UNSUPPORTED, "the graph has no weights");
    PC_TRY(use_device(g));
    if (vlist) PC_CUDA(cudaMemcpyAsync(vlist, g->off.p, (g->n + 1) * 8, cudaMemcpyDeviceToHost, g->stream));
    if (elist && g->m) PC_CUDA(cudaMemcpyAsync(elist, g->adj.p, g->m * 4, cudaMemcpyDeviceToHost, g->stream));
    if (weights && g->m) PC_CUDA(cudaMemcpyAsync(weights, g->w.p, g->m * 4, cudaMemcpyDeviceToHost, g->stream));
    PC_CUDA(cudaStreamSynchronize(g->stream));
    return PC_OK;
}

}  // extern "C"
