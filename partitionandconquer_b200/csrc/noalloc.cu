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
// kNoAllocMaxVertices vertices plus the total, the pivot counter and an error
// word, so graphs with more vertices are rejected.  All calls share it and it
// keeps the previous call's contents: each call clears the counters and the
// error word before use and writes dplus for its own n vertices only, and two
// calls whose work overlaps on the GPU (different streams, no ordering
// between them) race on it.
//
// The CSR is checked as far as memory safety needs: offsets must be
// non-decreasing and end at m, and every neighbour id that is dereferenced
// must lie in [0, n).  A violation sets the error word, the counting kernel
// does no work, and the call returns PC_ERR_INVALID_INPUT.
#include "pc_internal.cuh"
#include "tc_kernels.cuh"

namespace pc {
namespace na {

constexpr uint64_t kNoAllocMaxVertices = 1ull << 20;
constexpr int kWarps = 8;

// [0, kNoAllocMaxVertices): dplus; then the triangle total, the error word
// (adjacent, so one 16-byte copy returns both) and the pivot counter.
struct NoAllocScratch {
    uint32_t dplus[kNoAllocMaxVertices];
    unsigned long long total;
    unsigned long long error;  // 1: offsets not monotone / not ending at m; 2: neighbour id outside [0, n)
    unsigned long long next_pivot;
};

static __device__ __align__(256) NoAllocScratch g_scratch;

// Zeroes the total, the pivot counter and the error word (one thread, first
// launch of every call, so nothing a previous call left behind is read).
__global__ void k_na_clear(NoAllocScratch* __restrict__ s) {
    s->total = 0;
    s->error = 0;
    s->next_pivot = 0;
}

// dplus of every row, and the offset checks; it only ever sets the error word.
__global__ void k_na_prepare(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj, uint64_t n,
                             uint64_t m, NoAllocScratch* __restrict__ s) {
    const uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (u >= n) return;
    uint64_t lo = off[u], hi = off[u + 1];
    if (lo > hi || hi > m || (u + 1 == n && hi != m)) {
        s->dplus[u] = 0;
        atomicOr(&s->error, 1ull);
        return;
    }
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
    // every block reads the prepare kernel's verdict before any row access
    // (stream order makes it visible); the counting is skipped on a bad CSR
    if (*(volatile unsigned long long*)&s->error) return;
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
                if ((uint64_t)(uint32_t)c >= n) {
                    atomicOr(&s->error, 2ull);
                    continue;
                }
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
                if ((uint64_t)(uint32_t)c >= n) {
                    atomicOr(&s->error, 2ull);
                    continue;
                }
                cnt += merge_below(adj + off[c], s->dplus[c], nb, dp, b);
            }
        }
    }
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0 && cnt) atomicAdd(&s->total, cnt);
}

// Device address of g_scratch in the caller's current context.  It is looked
// up on every call (a cheap query that allocates nothing): a cached address
// would go stale after cudaDeviceReset or under another context made current
// by a driver-API caller, and the kernels would then write through it.
static pc_status scratch_address(NoAllocScratch** out) {
    void* p = nullptr;
    PC_CUDA(cudaGetSymbolAddress(&p, g_scratch));
    *out = static_cast<NoAllocScratch*>(p);
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
    PC_TRY(scratch_address(&s));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_na_clear<<<1, 1, 0, st>>>(s);
    PC_LAUNCHED();
    k_na_prepare<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(d_vlist, d_elist, n, m, s);
    PC_LAUNCHED();
    k_na_tc<<<(unsigned)(sm_count(device) * 8), kWarps * 32, 0, st>>>(d_vlist, d_elist, n, s);
    PC_LAUNCHED();
    unsigned long long res[2] = {0, 0};  // total, error
    PC_CUDA(cudaMemcpyAsync(res, &s->total, sizeof(res), cudaMemcpyDeviceToHost, st));
    PC_CUDA(cudaStreamSynchronize(st));
    if (res[1] & 1ull) return fail(PC_ERR_INVALID_INPUT, "CSR offsets are not non-decreasing or do not end at m");
    if (res[1] & 2ull) return fail(PC_ERR_INVALID_INPUT, "CSR holds a neighbour id outside [0, n)");
    *count = res[0];
    return PC_OK;
}

}  // extern "C"
