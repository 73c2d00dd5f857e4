// Triangle counting for callers that cannot allocate device memory.
//
// Some callers must not call cudaMalloc: a process whose device memory is
// already owned by another allocator (a framework's pool that reserved the
// GPU up front), a latency-bound path where an allocation may synchronise the
// device or take unbounded time, or a deployment that fixes its device
// footprint at start-up.  pc_tc_count_noalloc serves them: the caller passes
// its own device-resident CSR and a host result slot, and every temporary the
// kernel needs lives in the file-scope array below, which the library image
// carries (each GPU that loads libpc.so holds it until the process exits).
//
// The array holds the per-vertex prefix lengths |N(u) & [0,u)| for at most
// kNoAllocMaxVertices vertices plus two counters, so graphs with more
// vertices are rejected.  All calls share it and it keeps the previous call's
// contents: each call clears the counters before use, and two calls whose
// work overlaps on the GPU (different streams, no ordering between them)
// race on it.
#include <climits>
#include <mutex>

#include "pc_internal.cuh"
#include "tc_kernels.cuh"

namespace pc {
namespace na {

constexpr uint64_t kNoAllocMaxVertices = 1ull << 20;
constexpr int kWarps = 8;

// [0, kNoAllocMaxVertices): dplus; then the triangle total and the pivot counter.
struct NoAllocScratch {
    uint32_t dplus[kNoAllocMaxVertices];
    unsigned long long total;
    unsigned long long next_pivot;
};

static __device__ __align__(256) NoAllocScratch g_scratch;

__global__ void k_na_prepare(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj, uint64_t n,
                             NoAllocScratch* __restrict__ s) {
    const uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (u == 0) {
        s->total = 0;
        s->next_pivot = 0;
    }
    if (u >= n) return;
    uint64_t lo = off[u], hi = off[u + 1];
    const uint64_t b = lo;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (adj[mid] < (int32_t)u) lo = mid + 1; else hi = mid;
    }
    s->dplus[u] = (uint32_t)(lo - b);
}

// The warp-hash pivot kernel of the handle-based path, with its pivot queue
// and total in the static scratch: a warp takes a pivot b, hashes N+(b) into
// warp-private shared memory (a merge when |N+(b)| > 256) and scans every
// in-neighbour's prefix below b.
__global__ void __launch_bounds__(kWarps * 32) k_na_tc(const uint64_t* __restrict__ off,
                                                       const int32_t* __restrict__ adj, uint64_t n,
                                                       NoAllocScratch* __restrict__ s) {
    using namespace tc;
    __shared__ int32_t table[kWarps][kHashSlots];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t* T = table[w];
    for (int i = lane; i < kHashSlots; i += 32) T[i] = -1;
    __syncwarp();
    unsigned long long cnt = 0;
    for (;;) {
        unsigned long long q = 0;
        if (lane == 0) q = atomicAdd(&s->next_pivot, 1ull);
        q = __shfl_sync(0xffffffffu, q, 0);
        if (q >= n) break;
        const int32_t b = (int32_t)q;
        const uint64_t rb = off[b], re = off[b + 1];
        const uint32_t dp = s->dplus[b];
        if (dp == 0 || rb + dp == re) continue;
        const int32_t* nb = adj + rb;
        if (dp <= (uint32_t)kHashCap) {
            for (uint32_t k = lane; k < dp; k += 32) {
                const int32_t a = nb[k];
                uint32_t slot = hash_slot(a);
                while (atomicCAS(&T[slot], -1, a) != -1) slot = (slot + 1) & (kHashSlots - 1);
            }
            __syncwarp();
            for (uint64_t e = rb + dp + lane; e < re; e += 32) {
                const int32_t c = adj[e];
                const int32_t* row = adj + off[c];
                const uint32_t lim = s->dplus[c];
                for (uint32_t i = 0; i < lim; ++i) {
                    const int32_t a = row[i];
                    if (a >= b) break;
                    uint32_t slot = hash_slot(a);
                    int32_t key;
                    while ((key = T[slot]) != -1) {
                        if (key == a) { ++cnt; break; }
                        slot = (slot + 1) & (kHashSlots - 1);
                    }
                }
            }
            __syncwarp();
            for (int i = lane; i < kHashSlots; i += 32) T[i] = -1;
            __syncwarp();
        } else {
            for (uint64_t e = rb + dp + lane; e < re; e += 32) {
                const int32_t c = adj[e];
                cnt += merge_below(adj + off[c], s->dplus[c], nb, dp, b);
            }
        }
    }
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0 && cnt) atomicAdd(&s->total, cnt);
}

// Device address of g_scratch per device, resolved once with that device current.
static std::mutex g_mu;
static NoAllocScratch* g_addr[64];

static pc_status scratch_address(int device, NoAllocScratch** out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (device < 0 || device >= 64) return fail(PC_ERR_INVALID_INPUT, "device index out of range");
    if (!g_addr[device]) {
        void* p = nullptr;
        PC_CUDA(cudaGetSymbolAddress(&p, g_scratch));
        g_addr[device] = static_cast<NoAllocScratch*>(p);
    }
    *out = g_addr[device];
    return PC_OK;
}

}  // namespace na
}  // namespace pc

using namespace pc;
using namespace pc::na;

extern "C" {

pc_status pc_tc_count_noalloc(const uint64_t* d_vlist, const int32_t* d_elist, uint64_t n, uint64_t m, void* stream,
                              uint64_t* count) {
    clear_error();
    if (!d_vlist || (m && !d_elist) || !count) return fail(PC_ERR_INVALID_INPUT, "null argument");
    if (n > kNoAllocMaxVertices) {
        char buf[160];
        snprintf(buf, sizeof(buf), "graph has %llu vertices; the allocation-free path holds at most %llu",
                 (unsigned long long)n, (unsigned long long)kNoAllocMaxVertices);
        return fail(PC_ERR_INVALID_INPUT, buf);
    }
    *count = 0;
    if (n == 0 || m == 0) return PC_OK;
    int device = 0;
    PC_CUDA(cudaGetDevice(&device));
    NoAllocScratch* s = nullptr;
    PC_TRY(scratch_address(device, &s));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_na_prepare<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(d_vlist, d_elist, n, s);
    PC_LAUNCHED();
    k_na_tc<<<(unsigned)(sm_count(device) * 8), kWarps * 32, 0, st>>>(d_vlist, d_elist, n, s);
    PC_LAUNCHED();
    unsigned long long total = 0;
    PC_CUDA(cudaMemcpyAsync(&total, &s->total, sizeof(total), cudaMemcpyDeviceToHost, st));
    PC_CUDA(cudaStreamSynchronize(st));
    *count = total;
    return PC_OK;
}

}  // extern "C"
