// Many independent graphs in one launch: triangle counts per graph, LCC per
// vertex and BFS levels per vertex (from each graph's first vertex).
//
// The graphs are packed in one CSR arena with arena-wide vertex ids; graph g
// owns vertices [voff[g], voff[g+1]) and no edge joins two graphs, so the
// arena is one block-diagonal graph.  A single persistent kernel takes work
// items (graph, task) from a global counter, largest graphs first, and runs
// each item inside one CTA: no CTA ever waits for another, so the launch
// needs no grid-wide synchronisation.  The launch sequence (counter reset,
// output clears, the kernel, the result copies) is captured once into a CUDA
// graph and replayed by later calls; the schedule (threads per CTA, CTAs per
// SM, item order) comes from pc_batch_autotune.
#include <algorithm>
#include <climits>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "pc_internal.cuh"
#include "tc_kernels.cuh"

struct pc_batch {
    pc_graph* g = nullptr;  // the arena (validated by pc_graph_create)
    uint32_t G = 0;
    std::vector<uint64_t> voff;
    std::vector<uint64_t> gm;  // directed edges per graph
    pc::DevBuf d_voff, dplus, graph_of, ecnt, dist, q0, q1, tc, lcc, items, counter;
    uint64_t* h_tc = nullptr;  // pinned staging
    double* h_lcc = nullptr;
    int32_t* h_bfs = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t exec_key = ~0ull;
    int threads = 512, ctas_per_sm = 2, order = 0;
    uint32_t nitems = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace pc {
namespace bt {

enum Task : int { kTC = 0, kLCC = 1, kBFS = 2 };
constexpr int kMaxWarps = 16;
constexpr int kSlots = 512;  // per-warp hash: keys + positions
constexpr int kCap = 256;

__global__ void k_graph_of(const uint64_t* __restrict__ voff, int32_t* __restrict__ graph_of) {
    const uint64_t v0 = voff[blockIdx.x], v1 = voff[blockIdx.x + 1];
    for (uint64_t v = v0 + threadIdx.x; v < v1; v += blockDim.x) graph_of[v] = (int32_t)blockIdx.x;
}

__global__ void k_prepare(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                          const uint64_t* __restrict__ voff, const int32_t* __restrict__ graph_of, uint64_t n,
                          uint32_t* __restrict__ dplus, uint32_t* __restrict__ bad) {
    const uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (u >= n) return;
    const uint64_t b = off[u], e = off[u + 1];
    if (e > b) {
        const int32_t g = graph_of[u];
        if ((uint64_t)adj[b] < voff[g] || (uint64_t)adj[e - 1] >= voff[g + 1]) atomicOr(bad, 1u);
    }
    uint64_t lo = b, hi = e;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (adj[mid] < (int32_t)u) lo = mid + 1; else hi = mid;
    }
    dplus[u] = (uint32_t)(lo - b);
}

struct Args {
    const uint64_t* off;
    const int32_t* adj;
    const uint32_t* dplus;
    const uint64_t* voff;
    const int32_t* items;  // graph * 4 + task
    uint32_t nitems;
    uint32_t* counter;     // [0] next item
    unsigned long long* tc;
    uint32_t* ecnt;
    double* lcc;
    int32_t* dist;
    int32_t* q0;
    int32_t* q1;
};

__device__ __forceinline__ uint32_t lbound(const int32_t* __restrict__ p, uint32_t n, int32_t x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (p[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Triangle listing of one graph by one CTA.  Warps take pivots from a shared
// counter; a pivot's set N+(b) goes into a warp-private hash (key -> position
// in row b), lanes scan in-neighbour prefixes.  With `edges`, every triangle
// adds 1 to its three edges' oriented slots (for LCC); otherwise the CTA
// returns its count.
template <bool kEdges>
__device__ unsigned long long cta_triangles(const Args& A, uint64_t v0, uint64_t v1, int32_t* keys, int32_t* vals,
                                            uint32_t* s_next) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t* K = keys + w * kSlots;
    int32_t* V = vals + w * kSlots;
    for (int i = lane; i < kSlots; i += 32) K[i] = -1;
    __syncwarp();
    unsigned long long cnt = 0;
    for (;;) {
        uint32_t q = 0;
        if (lane == 0) q = atomicAdd(s_next, 1u);
        q = __shfl_sync(0xffffffffu, q, 0);
        const uint64_t b64 = v0 + q;
        if (b64 >= v1) break;
        const int32_t b = (int32_t)b64;
        const uint64_t rb = A.off[b], re = A.off[b + 1];
        const uint32_t dp = A.dplus[b];
        if (dp == 0 || rb + dp == re) continue;
        const bool hashed = dp <= (uint32_t)kCap;
        if (hashed) {
            for (uint32_t k = lane; k < dp; k += 32) {
                const int32_t a = A.adj[rb + k];
                uint32_t s = tc::hash_slot(a);
                while (atomicCAS(&K[s], -1, a) != -1) s = (s + 1) & (kSlots - 1);
                V[s] = (int32_t)k;
            }
            __syncwarp();
        }
        for (uint64_t e = rb + dp + lane; e < re; e += 32) {
            const int32_t c = A.adj[e];
            const uint64_t rc = A.off[c];
            const uint32_t lim = A.dplus[c];
            uint32_t pair = 0, i = 0;
            for (; i < lim; ++i) {
                const int32_t a = A.adj[rc + i];
                if (a >= b) break;
                int32_t pos = -1;
                if (hashed) {
                    uint32_t s = tc::hash_slot(a);
                    int32_t key;
                    while ((key = K[s]) != -1) {
                        if (key == a) { pos = V[s]; break; }
                        s = (s + 1) & (kSlots - 1);
                    }
                } else {
                    const uint32_t p = lbound(A.adj + rb, dp, a);
                    if (p < dp && A.adj[rb + p] == a) pos = (int32_t)p;
                }
                if (pos >= 0) {
                    ++pair;
                    if (kEdges) {
                        atomicAdd(&A.ecnt[rc + i], 1u);   // edge {c, a}
                        atomicAdd(&A.ecnt[rb + pos], 1u); // edge {b, a}
                    }
                }
            }
            cnt += pair;
            // the scan stopped at b itself (b is in N(c) below c)
            if (kEdges && pair && i < lim && A.adj[rc + i] == b) atomicAdd(&A.ecnt[rc + i], pair);  // edge {c, b}
        }
        if (hashed) {
            __syncwarp();
            for (int i = lane; i < kSlots; i += 32) K[i] = -1;
            __syncwarp();
        }
    }
    return cnt;
}

__device__ void cta_lcc_finalize(const Args& A, uint64_t v0, uint64_t v1) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint64_t u = v0 + w; u < v1; u += nw) {
        const uint64_t b = A.off[u], e = A.off[u + 1];
        const uint64_t du = e - b;
        unsigned long long sum = 0;
        for (uint64_t j = b + lane; j < e; j += 32) {
            const int32_t v = A.adj[j];
            if ((uint64_t)v < u) {
                sum += A.ecnt[j];
            } else {
                const uint64_t rv = A.off[v];
                sum += A.ecnt[rv + lbound(A.adj + rv, A.dplus[v], (int32_t)u)];
            }
        }
        for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        // src/Graph.cpp:833-838
        if (lane == 0) A.lcc[u] = du < 1 ? 0.0 : (double)sum / (double)(du * (du - 1));
    }
}

// Level-synchronous BFS of one graph by one CTA (warp per frontier vertex).
__device__ void cta_bfs(const Args& A, uint64_t v0, uint64_t v1, uint32_t* s_cnt) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint64_t v = v0 + threadIdx.x; v < v1; v += blockDim.x) A.dist[v] = INT_MAX;
    __syncthreads();
    if (threadIdx.x == 0) {
        A.dist[v0] = 0;
        A.q0[v0] = (int32_t)v0;
        s_cnt[0] = 1;
    }
    __syncthreads();
    int32_t* fq = A.q0 + v0;
    int32_t* nq = A.q1 + v0;
    for (int32_t level = 1;; ++level) {
        const uint32_t fn = s_cnt[0];
        __syncthreads();
        if (fn == 0) break;
        if (threadIdx.x == 0) s_cnt[1] = 0;
        __syncthreads();
        for (uint32_t i = w; i < fn; i += nw) {
            const int32_t u = fq[i];
            const uint64_t b = A.off[u], e = A.off[u + 1];
            for (uint64_t j0 = b; j0 < e; j0 += 32) {
                const uint64_t j = j0 + lane;
                bool won = false;
                int32_t v = 0;
                if (j < e) {
                    v = A.adj[j];
                    if (A.dist[v] == INT_MAX) won = atomicCAS(&A.dist[v], INT_MAX, level) == INT_MAX;
                }
                const unsigned m = __ballot_sync(0xffffffffu, won);
                if (m) {
                    uint32_t base = 0;
                    if (lane == 0) base = atomicAdd(&s_cnt[1], (uint32_t)__popc(m));
                    base = __shfl_sync(0xffffffffu, base, 0);
                    if (won) nq[base + __popc(m & ((1u << lane) - 1u))] = v;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_cnt[0] = s_cnt[1];
        int32_t* t = fq;
        fq = nq;
        nq = t;
        __syncthreads();
    }
    for (uint64_t v = v0 + threadIdx.x; v < v1; v += blockDim.x) {
        const int32_t d = A.dist[v];
        A.dist[v] = d == 0 ? -1 : d;  // rank[src] = -1 (src/Graph.cpp:1704)
    }
}

__global__ void __launch_bounds__(kMaxWarps * 32) k_batch(Args A) {
    extern __shared__ int32_t smem[];
    __shared__ uint32_t s_item, s_next, s_cnt[2];
    __shared__ unsigned long long s_sum;
    const int nw = blockDim.x >> 5;
    int32_t* keys = smem;
    int32_t* vals = smem + nw * kSlots;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            s_item = atomicAdd(&A.counter[0], 1u);
            s_next = 0;
            s_sum = 0;
        }
        __syncthreads();
        const uint32_t it = s_item;
        if (it >= A.nitems) break;
        const int32_t code = A.items[it];
        const int32_t g = code >> 2, task = code & 3;
        const uint64_t v0 = A.voff[g], v1 = A.voff[g + 1];
        if (task == kTC) {
            unsigned long long c = cta_triangles<false>(A, v0, v1, keys, vals, &s_next);
            for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
            if ((threadIdx.x & 31) == 0 && c) atomicAdd(&s_sum, c);
            __syncthreads();
            if (threadIdx.x == 0) A.tc[g] = s_sum;
        } else if (task == kLCC) {
            cta_triangles<true>(A, v0, v1, keys, vals, &s_next);
            __threadfence_block();
            __syncthreads();
            cta_lcc_finalize(A, v0, v1);
        } else {
            cta_bfs(A, v0, v1, s_cnt);
        }
    }
}

static uint64_t key_of(uint32_t tasks, int threads, int cps, int order) {
    return ((uint64_t)tasks << 32) | ((uint64_t)threads << 16) | ((uint64_t)cps << 8) | (uint64_t)order;
}

}  // namespace bt
}  // namespace pc

using namespace pc;
using namespace pc::bt;

static pc_status batch_build_items(pc_batch* b, uint32_t tasks) {
    // largest graphs first (order 0) or graph order (order 1); LCC before TC
    // before BFS for one graph size.
    std::vector<int32_t> items;
    std::vector<uint32_t> gidx(b->G);
    std::iota(gidx.begin(), gidx.end(), 0u);
    if (b->order == 0)
        std::stable_sort(gidx.begin(), gidx.end(), [&](uint32_t x, uint32_t y) { return b->gm[x] > b->gm[y]; });
    for (uint32_t gi : gidx) {
        if (tasks & PC_BATCH_LCC) items.push_back((int32_t)(gi * 4 + kLCC));
        if (tasks & PC_BATCH_TC) items.push_back((int32_t)(gi * 4 + kTC));
        if (tasks & PC_BATCH_BFS) items.push_back((int32_t)(gi * 4 + kBFS));
    }
    b->nitems = (uint32_t)items.size();
    PC_TRY(b->items.ensure(std::max<size_t>(items.size(), 1) * 4, "batch items"));
    if (!items.empty())
        PC_CUDA(cudaMemcpyAsync(b->items.p, items.data(), items.size() * 4, cudaMemcpyHostToDevice, b->g->stream));
    PC_CUDA(cudaStreamSynchronize(b->g->stream));
    return PC_OK;
}

static pc_status batch_capture(pc_batch* b, uint32_t tasks) {
    const uint64_t key = key_of(tasks, b->threads, b->ctas_per_sm, b->order);
    if (b->exec && b->exec_key == key) return PC_OK;
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    PC_TRY(batch_build_items(b, tasks));
    cudaStream_t s = b->g->stream;
    const uint64_t N = b->g->n, M = b->g->m;
    Args A;
    A.off = b->g->off.as<uint64_t>();
    A.adj = b->g->adj.as<int32_t>();
    A.dplus = b->dplus.as<uint32_t>();
    A.voff = b->d_voff.as<uint64_t>();
    A.items = b->items.as<int32_t>();
    A.nitems = b->nitems;
    A.counter = b->counter.as<uint32_t>();
    A.tc = b->tc.as<unsigned long long>();
    A.ecnt = b->ecnt.as<uint32_t>();
    A.lcc = b->lcc.as<double>();
    A.dist = b->dist.as<int32_t>();
    A.q0 = b->q0.as<int32_t>();
    A.q1 = b->q1.as<int32_t>();
    const int nw = b->threads / 32;
    const size_t smem = (size_t)nw * kSlots * 4 * 2;
    PC_CUDA(cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const unsigned grid = (unsigned)(sm_count(b->g->device) * b->ctas_per_sm);
    PC_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(b->counter.p, 0, 16, s);
    if (tasks & PC_BATCH_TC) cudaMemsetAsync(b->tc.p, 0, (size_t)b->G * 8, s);
    if (tasks & PC_BATCH_LCC) cudaMemsetAsync(b->ecnt.p, 0, std::max<uint64_t>(M, 1) * 4, s);
    k_batch<<<grid, b->threads, smem, s>>>(A);
    if (tasks & PC_BATCH_TC) cudaMemcpyAsync(b->h_tc, b->tc.p, (size_t)b->G * 8, cudaMemcpyDeviceToHost, s);
    if (tasks & PC_BATCH_LCC) cudaMemcpyAsync(b->h_lcc, b->lcc.p, N * 8, cudaMemcpyDeviceToHost, s);
    if (tasks & PC_BATCH_BFS) cudaMemcpyAsync(b->h_bfs, b->dist.p, N * 4, cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamEndCapture(s, &b->graph);
    if (e != cudaSuccess) return cuda_fail(e, "stream capture of the batch launch", __FILE__, __LINE__);
    PC_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
    b->exec_key = key;
    return PC_OK;
}

extern "C" {

pc_status pc_batch_create(const uint64_t* vlist, const int32_t* elist, uint64_t N, uint64_t M, const uint64_t* voff,
                          uint32_t G, pc_batch** out) {
    clear_error();
    if (!out || !voff || G == 0) return fail(PC_ERR_INVALID_INPUT, "bad argument");
    *out = nullptr;
    if (voff[0] != 0 || voff[G] != N) return fail(PC_ERR_INVALID_INPUT, "graph offsets must run from 0 to N");
    for (uint32_t g = 0; g < G; ++g)
        if (voff[g + 1] <= voff[g]) return fail(PC_ERR_INVALID_INPUT, "every graph needs at least one vertex");
    pc_graph* arena = nullptr;
    PC_TRY(pc_graph_create(vlist, elist, nullptr, N, M, 0, &arena));
    pc_batch* b = new pc_batch();
    b->g = arena;
    b->G = G;
    b->voff.assign(voff, voff + G + 1);
    b->gm.resize(G);
    for (uint32_t g = 0; g < G; ++g) b->gm[g] = vlist[voff[g + 1]] - vlist[voff[g]];
    auto bail = [&](pc_status st) {
        const std::string msg = pc_last_error();  // pc_graph_destroy clears it
        if (b->h_tc) cudaFreeHost(b->h_tc);
        if (b->h_lcc) cudaFreeHost(b->h_lcc);
        if (b->h_bfs) cudaFreeHost(b->h_bfs);
        pc_graph_destroy(b->g);
        delete b;
        return fail(st, msg);
    };
    pc_status st;
    if ((st = b->d_voff.alloc((G + 1) * 8, "graph offsets")) != PC_OK || (st = b->dplus.alloc(N * 4, "dplus")) != PC_OK ||
        (st = b->graph_of.alloc(N * 4, "graph of vertex")) != PC_OK ||
        (st = b->ecnt.alloc(std::max<uint64_t>(M, 1) * 4, "edge counts")) != PC_OK ||
        (st = b->dist.alloc(N * 4, "levels")) != PC_OK || (st = b->q0.alloc(N * 4, "queue")) != PC_OK ||
        (st = b->q1.alloc(N * 4, "queue")) != PC_OK || (st = b->tc.alloc((size_t)G * 8, "counts")) != PC_OK ||
        (st = b->lcc.alloc(N * 8, "lcc")) != PC_OK || (st = b->counter.alloc(16, "counter")) != PC_OK)
        return bail(st);
    cudaError_t e = cudaMallocHost(&b->h_tc, (size_t)G * 8);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_lcc, N * 8);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_bfs, N * 4);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
    if (e != cudaSuccess) return bail(cuda_fail(e, "pinned staging", __FILE__, __LINE__));
    cudaStream_t s = arena->stream;
    DevBuf chk;
    if ((st = chk.alloc(16, "check")) != PC_OK) return bail(st);
    e = cudaMemcpyAsync(b->d_voff.p, voff, (G + 1) * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(chk.p, 0, 16, s);
    if (e != cudaSuccess) return bail(cuda_fail(e, "batch upload", __FILE__, __LINE__));
    k_graph_of<<<G, 256, 0, s>>>(b->d_voff.as<uint64_t>(), b->graph_of.as<int32_t>());
    count_launch();
    k_prepare<<<(unsigned)ceil_div(N, 256), 256, 0, s>>>(arena->off.as<uint64_t>(), arena->adj.as<int32_t>(),
                                                         b->d_voff.as<uint64_t>(), b->graph_of.as<int32_t>(), N,
                                                         b->dplus.as<uint32_t>(), chk.as<uint32_t>());
    count_launch();
    uint32_t bad = 0;
    e = cudaMemcpyAsync(&bad, chk.p, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return bail(cuda_fail(e, "batch preparation", __FILE__, __LINE__));
    if (bad) return bail(fail(PC_ERR_INVALID_INPUT, "an edge joins two graphs of the batch"));
    *out = b;
    return PC_OK;
}

pc_status pc_batch_destroy(pc_batch* b) {
    clear_error();
    if (!b) return PC_OK;
    cudaSetDevice(b->g->device);
    cudaStreamSynchronize(b->g->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->h_tc) cudaFreeHost(b->h_tc);
    if (b->h_lcc) cudaFreeHost(b->h_lcc);
    if (b->h_bfs) cudaFreeHost(b->h_bfs);
    pc_graph* g = b->g;
    delete b;
    return pc_graph_destroy(g);
}

pc_status pc_batch_set_schedule(pc_batch* b, int32_t threads, int32_t ctas_per_sm, int32_t order) {
    clear_error();
    if (!b) return fail(PC_ERR_INVALID_INPUT, "null batch");
    if ((threads != 256 && threads != 512) || ctas_per_sm < 1 || ctas_per_sm > 4 || (order != 0 && order != 1))
        return fail(PC_ERR_INVALID_INPUT, "schedule: threads 256|512, ctas_per_sm 1..4, order 0|1");
    b->threads = threads;
    b->ctas_per_sm = ctas_per_sm;
    b->order = order;
    return PC_OK;
}

pc_status pc_batch_run(pc_batch* b, uint32_t tasks, uint64_t* tc, double* lcc, int32_t* bfs, pc_batch_stats* stats) {
    clear_error();
    if (!b || !tasks || (tasks & ~7u)) return fail(PC_ERR_INVALID_INPUT, "bad argument");
    if (((tasks & PC_BATCH_TC) && !tc) || ((tasks & PC_BATCH_LCC) && !lcc) || ((tasks & PC_BATCH_BFS) && !bfs))
        return fail(PC_ERR_INVALID_INPUT, "missing output buffer");
    PC_TRY(use_device(b->g));
    PC_TRY(batch_capture(b, tasks));
    cudaStream_t s = b->g->stream;
    PC_CUDA(cudaEventRecord(b->ev0, s));
    PC_CUDA(cudaGraphLaunch(b->exec, s));
    PC_CUDA(cudaEventRecord(b->ev1, s));
    PC_CUDA(cudaStreamSynchronize(s));
    PC_CUDA(cudaGetLastError());
    count_launch();
    const uint64_t N = b->g->n;
    if (tasks & PC_BATCH_TC) memcpy(tc, b->h_tc, (size_t)b->G * 8);
    if (tasks & PC_BATCH_LCC) memcpy(lcc, b->h_lcc, N * 8);
    if (tasks & PC_BATCH_BFS) memcpy(bfs, b->h_bfs, N * 4);
    if (stats) {
        float ms = 0.f;
        PC_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
        stats->ms = ms;
        stats->items = b->nitems;
        stats->threads = b->threads;
        stats->ctas_per_sm = b->ctas_per_sm;
        stats->order = b->order;
    }
    return PC_OK;
}

pc_status pc_batch_autotune(pc_batch* b, uint32_t tasks, pc_batch_stats* best) {
    clear_error();
    if (!b) return fail(PC_ERR_INVALID_INPUT, "null batch");
    const uint64_t N = b->g->n;
    std::vector<uint64_t> tc(b->G);
    std::vector<double> lcc(N);
    std::vector<int32_t> bfs(N);
    double best_ms = 1e30;
    int bt = b->threads, bc = b->ctas_per_sm, bo = b->order;
    const int thr[] = {256, 512};
    for (int t : thr)
        for (int c = 1; c <= 4; c *= 2)
            for (int o = 0; o < 2; ++o) {
                if (t == 512 && c > 2) continue;
                PC_TRY(pc_batch_set_schedule(b, t, c, o));
                pc_batch_stats st;
                PC_TRY(pc_batch_run(b, tasks, tc.data(), lcc.data(), bfs.data(), &st));  // warm / capture
                PC_TRY(pc_batch_run(b, tasks, tc.data(), lcc.data(), bfs.data(), &st));
                if (st.ms < best_ms) {
                    best_ms = st.ms;
                    bt = t;
                    bc = c;
                    bo = o;
                }
            }
    PC_TRY(pc_batch_set_schedule(b, bt, bc, bo));
    if (best) {
        PC_TRY(pc_batch_run(b, tasks, tc.data(), lcc.data(), bfs.data(), best));
    }
    return PC_OK;
}

}  // extern "C"
