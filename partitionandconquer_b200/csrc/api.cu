// Library plumbing of libpc.so: errors, device selection, graph upload with
// device-side validation, the partitioned view, reorder and layout export.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "pc_internal.cuh"

namespace pc {

// ---- errors ----------------------------------------------------------------

static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }
pc_status fail(pc_status st, const std::string& msg) {
    set_error(msg);
    return st;
}
pc_status cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
    char buf[512];
    snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what, file, line);
    if (e == cudaErrorMemoryAllocation) return fail(PC_ERR_OOM, buf);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return fail(PC_ERR_NO_DEVICE, buf);
    return fail(PC_ERR_CUDA, buf);
}
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// ---- memory ----------------------------------------------------------------

// Device buffers come from the device's default stream-ordered memory pool,
// whose release threshold is raised once per device so that freed blocks stay
// cached in the process: creating and destroying graph handles again and
// again (one upload per call of a drop-in caller) then reuses memory instead
// of mapping and unmapping it each time.  pc_release_cached_memory() trims the
// pools.  An allocation completes before alloc() returns (the legacy stream
// is synchronised), and release() waits for the device to go idle before the
// block returns to the pool, so no stream still uses it.
static std::mutex g_pool_mu;
static std::vector<int> g_pool_ready;

static cudaError_t prepare_pool(int dev) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if ((int)g_pool_ready.size() <= dev) g_pool_ready.resize(dev + 1, 0);
    if (g_pool_ready[dev]) return cudaSuccess;
    cudaMemPool_t pool;
    cudaError_t e = cudaDeviceGetDefaultMemPool(&pool, dev);
    if (e != cudaSuccess) return e;
    uint64_t keep = ~0ull;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e == cudaSuccess) g_pool_ready[dev] = 1;
    return e;
}

pc_status DevBuf::alloc(size_t nbytes, const char* what) {
    release();
    if (nbytes == 0) return PC_OK;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = prepare_pool(dev);
    if (e == cudaSuccess) e = cudaMallocAsync(&p, nbytes, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
        p = nullptr;
        cudaGetLastError();
        char buf[256];
        snprintf(buf, sizeof(buf), "device allocation of %zu bytes for %s failed: %s", nbytes, what, cudaGetErrorString(e));
        return fail(e == cudaErrorMemoryAllocation ? PC_ERR_OOM : PC_ERR_CUDA, buf);
    }
    bytes = nbytes;
    return PC_OK;
}
pc_status DevBuf::ensure(size_t nbytes, const char* what) {
    if (nbytes <= bytes) return PC_OK;
    return alloc(nbytes, what);
}
void DevBuf::release() {
    if (p) {
        int cur = -1;
        cudaGetDevice(&cur);
        if (cur != dev) cudaSetDevice(dev);
        cudaDeviceSynchronize();
        cudaFreeAsync(p, 0);
        cudaStreamSynchronize(0);
        if (cur != dev && cur >= 0) cudaSetDevice(cur);
    }
    p = nullptr;
    bytes = 0;
}

int sm_count(int device) {
    static std::mutex mu;
    static std::vector<int> cache;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)cache.size() <= device) cache.resize(device + 1, 0);
    if (!cache[device]) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) v = 148;
        cache[device] = v;
    }
    return cache[device];
}

pc_status use_device(const pc_graph* g) {
    PC_CUDA(cudaSetDevice(g->device));
    return PC_OK;
}

pc_status scratch_reserve(pc_pgraph* pg, size_t bytes) {
    pg->scratch.reset();
    // room for alignment padding of up to 64 sub-regions
    size_t want = bytes + 64 * 256;
    if (want > pg->scratch.buf.bytes) {
        PC_CUDA(cudaStreamSynchronize(pg->g->stream));
        PC_TRY(pg->scratch.buf.alloc(want + want / 4, "scratch arena"));
    }
    return PC_OK;
}

pc_status sync(pc_pgraph* pg) {
    PC_CUDA(cudaStreamSynchronize(pg->g->stream));
    PC_CUDA(cudaGetLastError());
    return PC_OK;
}

// ---- kernels: validation -----------------------------------------------------

enum : uint32_t {
    BAD_OFFSETS = 1u,
    BAD_RANGE = 2u,
    BAD_ORDER = 4u,
    BAD_SELF = 8u,
    BAD_WEIGHT = 16u,
};

__global__ void k_check_offsets(const uint64_t* __restrict__ off, uint64_t n, uint64_t m, uint32_t* err) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) {
        uint64_t a = off[i], b = off[i + 1];
        if (b < a || b > m) atomicOr(err, BAD_OFFSETS);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && (off[0] != 0 || off[n] != m)) atomicOr(err, BAD_OFFSETS);
}

// Warp-chunked edge walk: each warp takes a chunk of 1024 consecutive edge
// slots; lane 0 finds the row of the chunk start by binary search, then lanes
// walk forward to the row of their own slot.
__device__ __forceinline__ uint64_t row_of(const uint64_t* __restrict__ off, uint64_t n, uint64_t e) {
    uint64_t lo = 0, hi = n;  // off[lo] <= e < off[hi]
    while (hi - lo > 1) {
        uint64_t mid = (lo + hi) >> 1;
        if (off[mid] <= e) lo = mid; else hi = mid;
    }
    return lo;
}

// Symmetry fingerprint: each directed entry (u, v) adds +H(min, max) if u < v
// and -H(min, max) if u > v; a symmetric edge multiset sums to zero.  Two
// independent 64-bit hashes make a false "symmetric" verdict ~2^-128.
__device__ __forceinline__ uint64_t fp_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__global__ void k_check_edges(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj, uint64_t n,
                              uint64_t m, uint32_t* err, unsigned long long* fp) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    uint64_t acc0 = 0, acc1 = 0;
    uint32_t bad = 0;
    for (uint64_t c = warp; c * 1024 < m; c += nwarps) {
        uint64_t base = c * 1024, end = min(base + 1024, m);
        uint64_t r = 0;
        if (lane == 0) r = row_of(off, n, base);
        r = __shfl_sync(0xffffffffu, r, 0);
        for (uint64_t e0 = base; e0 < end; e0 += 32) {
            uint64_t e = e0 + lane;
            uint64_t u = r;
            if (e < end) {
                while (off[u + 1] <= e) ++u;
                int32_t v = adj[e];
                if (v < 0 || (uint64_t)v >= n) {
                    bad |= BAD_RANGE;
                } else {
                    if ((uint64_t)v == u) bad |= BAD_SELF;
                    if (e > off[u] && adj[e - 1] >= v) bad |= BAD_ORDER;
                    const uint64_t uv = (uint64_t)v;
                    const uint64_t lo = u < uv ? u : uv, hi = u < uv ? uv : u;
                    uint64_t key = (lo << 32) | hi;
                    uint64_t h0 = fp_mix(key ^ 0x243F6A8885A308D3ULL), h1 = fp_mix(key + 0x13198A2E03707344ULL);
                    if (u < (uint64_t)v) { acc0 += h0; acc1 += h1; } else { acc0 -= h0; acc1 -= h1; }
                }
            }
            r = __shfl_sync(0xffffffffu, u, 31);
        }
    }
    for (int o = 16; o; o >>= 1) {
        acc0 += __shfl_xor_sync(0xffffffffu, acc0, o);
        acc1 += __shfl_xor_sync(0xffffffffu, acc1, o);
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if (lane == 0) {
        if (acc0) atomicAdd(&fp[0], (unsigned long long)acc0);
        if (acc1) atomicAdd(&fp[1], (unsigned long long)acc1);
        if (bad) atomicOr(err, bad);
    }
}

// Weights must be in [0, 2^30): non-negative for the shortest-path semantics,
// and small enough that a distance plus a weight cannot overflow int32.
__global__ void k_check_weights(const int32_t* __restrict__ w, uint64_t m, uint32_t* err) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    bool bad = false;
    for (; i < m; i += stride) bad |= (w[i] < 0 || w[i] >= (1 << 30));
    if (bad) atomicOr(err, BAD_WEIGHT);
}

// ---- kernels: partition layout export ---------------------------------------

__global__ void k_layout_count(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                               const int32_t* __restrict__ v2p, const int32_t* __restrict__ api2int, uint64_t n,
                               uint64_t* __restrict__ cnt) {
    uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    uint64_t u = api2int ? (uint64_t)api2int[r] : r;
    for (uint64_t e = off[u]; e < off[u + 1]; ++e) cnt[(uint64_t)v2p[adj[e]] * n + r] += 1;
}

__global__ void k_layout_fill(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj,
                              const int32_t* __restrict__ w, const int32_t* __restrict__ v2p,
                              const int32_t* __restrict__ api2int, const int32_t* __restrict__ int2api, uint64_t n,
                              uint64_t* __restrict__ pos, int32_t* __restrict__ out_e, int32_t* __restrict__ out_w) {
    uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    uint64_t u = api2int ? (uint64_t)api2int[r] : r;
    for (uint64_t e = off[u]; e < off[u + 1]; ++e) {
        int32_t v = adj[e];
        uint64_t slot = (uint64_t)v2p[v] * n + r;
        uint64_t p = pos[slot]++;
        out_e[p] = int2api ? int2api[v] : v;
        if (out_w) out_w[p] = w[e];
    }
}

__global__ void k_dplus(const uint64_t* __restrict__ off, const int32_t* __restrict__ adj, uint64_t n,
                        uint32_t* __restrict__ dplus) {
    uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (u >= n) return;
    uint64_t lo = off[u], hi = off[u + 1], b = lo;
    // lower_bound(N(u), u)
    while (lo < hi) {
        uint64_t mid = (lo + hi) >> 1;
        if (adj[mid] < (int32_t)u) lo = mid + 1; else hi = mid;
    }
    dplus[u] = (uint32_t)(lo - b);
}

template <class T>
__global__ void k_gather(const T* __restrict__ in, const int32_t* __restrict__ idx, uint64_t n, T* __restrict__ out) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[idx[i]];
}

// Partition vector checks: stats[0] |= 1 on a negative id, stats[1] = max
// id, stats[2] |= 1 where v2p decreases (then partitions are not contiguous
// id ranges).
__global__ void k_v2p_stats(const int32_t* __restrict__ v2p, uint64_t n, int32_t* __restrict__ stats) {
    int32_t mx = 0, neg = 0, dec = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += stride) {
        const int32_t k = v2p[u];
        neg |= k < 0;
        mx = max(mx, k);
        if (u && k < v2p[u - 1]) dec = 1;
    }
    for (int o = 16; o; o >>= 1) {
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        neg |= __shfl_xor_sync(0xffffffffu, neg, o);
        dec |= __shfl_xor_sync(0xffffffffu, dec, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (neg) atomicOr(&stats[0], 1);
        atomicMax(&stats[1], mx);
        if (dec) atomicOr(&stats[2], 1);
    }
}

// pstart[k] = first position whose (non-decreasing) partition id is >= k.
__global__ void k_partition_starts(const int32_t* __restrict__ key, uint64_t n, int64_t P, int64_t* __restrict__ pstart) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= n; i += stride) {
        const int64_t cur = i < n ? key[i] : P;
        const int64_t prev = i == 0 ? -1 : key[i - 1];
        for (int64_t k = prev + 1; k <= cur; ++k) pstart[k] = (int64_t)i;
    }
}

__global__ void k_iota_i32(int32_t* __restrict__ a, uint64_t n) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) a[i] = (int32_t)i;
}

__global__ void k_invert(const int32_t* __restrict__ new2old, uint64_t n, int32_t* __restrict__ old2new) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) old2new[new2old[i]] = (int32_t)i;
}

__global__ void k_map_ids(int32_t* ids, const int32_t* __restrict__ map, uint64_t count) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < count) ids[i] = map[ids[i]];
}

// ---- id maps -----------------------------------------------------------------

bool api_is_internal(const pc_pgraph* pg) { return !pg->reordered_view || pg->contiguous; }

pc_status map_ids_to_internal(pc_pgraph* pg, int32_t* d_ids, uint64_t count) {
    if (api_is_internal(pg) || count == 0) return PC_OK;
    k_map_ids<<<(unsigned)ceil_div(count, 256), 256, 0, pg->g->stream>>>(d_ids, pg->new2old.as<int32_t>(), count);
    PC_LAUNCHED();
    return PC_OK;
}

template <class T>
static pc_status gather_to_api(pc_pgraph* pg, const T* in, T* out) {
    uint64_t n = pg->g->n;
    if (api_is_internal(pg)) {
        if (in != out) PC_CUDA(cudaMemcpyAsync(out, in, n * sizeof(T), cudaMemcpyDeviceToDevice, pg->g->stream));
        return PC_OK;
    }
    // out[api id a] = in[internal id of a] = in[new2old[a]]
    k_gather<T><<<(unsigned)ceil_div(n, 256), 256, 0, pg->g->stream>>>(in, pg->new2old.as<int32_t>(), n, out);
    PC_LAUNCHED();
    return PC_OK;
}
pc_status gather_to_api_i32(pc_pgraph* pg, const int32_t* in, int32_t* out) { return gather_to_api(pg, in, out); }
pc_status gather_to_api_f32(pc_pgraph* pg, const float* in, float* out) { return gather_to_api(pg, in, out); }
pc_status gather_to_api_f64(pc_pgraph* pg, const double* in, double* out) { return gather_to_api(pg, in, out); }

template <class T>
static pc_status gather_to_internal(pc_pgraph* pg, const T* in, T* out) {
    uint64_t n = pg->g->n;
    if (api_is_internal(pg)) {
        if (in != out) PC_CUDA(cudaMemcpyAsync(out, in, n * sizeof(T), cudaMemcpyDeviceToDevice, pg->g->stream));
        return PC_OK;
    }
    // out[internal u] = in[API id of u] = in[old2new[u]]
    k_gather<T><<<(unsigned)ceil_div(n, 256), 256, 0, pg->g->stream>>>(in, pg->old2new.as<int32_t>(), n, out);
    PC_LAUNCHED();
    return PC_OK;
}
pc_status gather_to_internal_i32(pc_pgraph* pg, const int32_t* in, int32_t* out) { return gather_to_internal(pg, in, out); }
pc_status gather_to_internal_f32(pc_pgraph* pg, const float* in, float* out) { return gather_to_internal(pg, in, out); }
pc_status gather_to_internal_f64(pc_pgraph* pg, const double* in, double* out) { return gather_to_internal(pg, in, out); }

int32_t to_internal_id(const pc_pgraph* pg, int32_t api_id) {
    if (api_is_internal(pg)) return api_id;
    int32_t v = 0;
    cudaMemcpy(&v, pg->new2old.as<int32_t>() + api_id, 4, cudaMemcpyDeviceToHost);
    return v;
}

pc_status ensure_dplus(pc_pgraph* pg) {
    if (pg->dplus.p) return PC_OK;
    uint64_t n = pg->g->n;
    PC_TRY(pg->dplus.alloc(std::max<uint64_t>(n, 1) * sizeof(uint32_t), "dplus"));
    if (n) {
        k_dplus<<<(unsigned)ceil_div(n, 256), 256, 0, pg->g->stream>>>(pg->off, pg->adj, n, pg->dplus.as<uint32_t>());
        PC_LAUNCHED();
    }
    return PC_OK;
}

}  // namespace pc

using namespace pc;

// ---- C ABI -------------------------------------------------------------------

extern "C" {

const char* pc_last_error(void) { return g_last_error.c_str(); }

pc_status pc_release_cached_memory(void) {
    clear_error();
    std::lock_guard<std::mutex> lk(g_pool_mu);
    for (int d = 0; d < (int)g_pool_ready.size(); ++d) {
        if (!g_pool_ready[d]) continue;
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, d) != cudaSuccess) continue;
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(d);
        cudaDeviceSynchronize();
        const cudaError_t e = cudaMemPoolTrimTo(pool, 0);
        cudaSetDevice(cur);
        if (e != cudaSuccess) return cuda_fail(e, "memory pool trim", __FILE__, __LINE__);
    }
    return PC_OK;
}
const char* pc_version(void) { return "pc-b200 0.1 (sm_100a)"; }

int32_t pc_device_count(void) {
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return c;
}

pc_status pc_set_device(int32_t device) {
    clear_error();
    int c = pc_device_count();
    if (c == 0) return fail(PC_ERR_NO_DEVICE, "no CUDA device is visible");
    if (device < 0 || device >= c) return fail(PC_ERR_INVALID_INPUT, "device index out of range");
    PC_CUDA(cudaSetDevice(device));
    return PC_OK;
}

uint64_t pc_launch_count(void) { return g_launches.load(); }

pc_status pc_host_register(void* ptr, size_t bytes) {
    clear_error();
    if (!ptr || !bytes) return fail(PC_ERR_INVALID_INPUT, "null or empty host buffer");
    if (pc_device_count() == 0) return fail(PC_ERR_NO_DEVICE, "no CUDA device is visible");
    PC_CUDA(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
    return PC_OK;
}

pc_status pc_host_unregister(void* ptr) {
    clear_error();
    if (!ptr) return fail(PC_ERR_INVALID_INPUT, "null host buffer");
    PC_CUDA(cudaHostUnregister(ptr));
    return PC_OK;
}

pc_status pc_graph_create(const uint64_t* vlist, const int32_t* elist, const int32_t* weights, uint64_t n,
                          uint64_t m, uint32_t flags, pc_graph** out) {
    clear_error();
    if (!out) return fail(PC_ERR_INVALID_INPUT, "out is null");
    *out = nullptr;
    if (!vlist) return fail(PC_ERR_INVALID_INPUT, "csr_vlist is null");
    if (m && !elist) return fail(PC_ERR_INVALID_INPUT, "csr_elist is null");
    if (n >= (1ull << 31)) return fail(PC_ERR_INVALID_INPUT, "vertex count exceeds the int32 id range");
    if (pc_device_count() == 0) return fail(PC_ERR_NO_DEVICE, "no CUDA device is visible");
    pc_graph* g = new pc_graph();
    auto cleanup = [&](pc_status s) {
        if (g->stream) cudaStreamDestroy(g->stream);
        delete g;
        return s;
    };
    cudaError_t e = cudaGetDevice(&g->device);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaGetDevice", __FILE__, __LINE__));
    e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaStreamCreate", __FILE__, __LINE__));
    g->n = n;
    g->m = m;
    g->weighted = weights != nullptr;
    pc_status st;
    if ((st = g->off.alloc((n + 1) * sizeof(uint64_t), "csr_vlist")) != PC_OK) return cleanup(st);
    // 64 padding ids: kernels may read a few slots past a row end (never used).
    if ((st = g->adj.alloc((m + 64) * sizeof(int32_t), "csr_elist")) != PC_OK) return cleanup(st);
    if (g->weighted && (st = g->w.alloc(std::max<uint64_t>(m, 1) * sizeof(int32_t), "csr_weight")) != PC_OK)
        return cleanup(st);
    e = cudaMemcpyAsync(g->off.p, vlist, (n + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, g->stream);
    if (e == cudaSuccess && m)
        e = cudaMemcpyAsync(g->adj.p, elist, m * sizeof(int32_t), cudaMemcpyHostToDevice, g->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(g->adj.as<int32_t>() + m, 0x7f, 64 * sizeof(int32_t), g->stream);
    if (e == cudaSuccess && g->weighted && m)
        e = cudaMemcpyAsync(g->w.p, weights, m * sizeof(int32_t), cudaMemcpyHostToDevice, g->stream);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "upload of the CSR", __FILE__, __LINE__));
    if (!(flags & PC_GRAPH_NO_VALIDATE)) {
        DevBuf chk;
        if ((st = chk.alloc(64, "validation words")) != PC_OK) return cleanup(st);
        uint32_t* d_err = chk.as<uint32_t>();
        unsigned long long* d_fp = reinterpret_cast<unsigned long long*>(chk.as<char>() + 16);
        e = cudaMemsetAsync(chk.p, 0, 64, g->stream);
        if (e != cudaSuccess) return cleanup(cuda_fail(e, "memset", __FILE__, __LINE__));
        int sms = sm_count(g->device);
        k_check_offsets<<<sms * 4, 256, 0, g->stream>>>(g->off.as<uint64_t>(), n, m, d_err);
        count_launch();
        uint32_t h_err = 0;
        e = cudaMemcpyAsync(&h_err, d_err, 4, cudaMemcpyDeviceToHost, g->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
        if (e != cudaSuccess) return cleanup(cuda_fail(e, "offset validation", __FILE__, __LINE__));
        if (h_err) return cleanup(fail(PC_ERR_INVALID_INPUT, "csr_vlist must start at 0, be non-decreasing and end at m"));
        if (m) {
            k_check_edges<<<sms * 8, 256, 0, g->stream>>>(g->off.as<uint64_t>(), g->adj.as<int32_t>(), n, m, d_err, d_fp);
            count_launch();
            if (g->weighted) {
                k_check_weights<<<sms * 4, 256, 0, g->stream>>>(g->w.as<int32_t>(), m, d_err);
                count_launch();
            }
        }
        uint64_t h_fp[2] = {0, 0};
        e = cudaMemcpyAsync(&h_err, d_err, 4, cudaMemcpyDeviceToHost, g->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_fp, d_fp, 16, cudaMemcpyDeviceToHost, g->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
        if (e != cudaSuccess) return cleanup(cuda_fail(e, "edge validation", __FILE__, __LINE__));
        if (h_err & BAD_RANGE) return cleanup(fail(PC_ERR_INVALID_INPUT, "csr_elist holds a vertex id outside [0, n)"));
        if (h_err & BAD_SELF) return cleanup(fail(PC_ERR_INVALID_INPUT, "csr_elist holds a self-loop"));
        if (h_err & BAD_ORDER)
            return cleanup(fail(PC_ERR_INVALID_INPUT, "neighbour lists must be strictly ascending (sorted, no duplicates)"));
        if (h_fp[0] || h_fp[1]) return cleanup(fail(PC_ERR_INVALID_INPUT, "the adjacency is not symmetric"));
        if (h_err & BAD_WEIGHT) return cleanup(fail(PC_ERR_INVALID_INPUT, "edge weights must be in [0, 2^30)"));
    } else {
        e = cudaStreamSynchronize(g->stream);
        if (e != cudaSuccess) return cleanup(cuda_fail(e, "upload", __FILE__, __LINE__));
    }
    *out = g;
    return PC_OK;
}

pc_status pc_graph_destroy(pc_graph* g) {
    clear_error();
    if (!g) return PC_OK;
    if (g->live_views) return fail(PC_ERR_INVALID_INPUT, "destroy the partitioned views of this graph first");
    cudaSetDevice(g->device);
    cudaStreamSynchronize(g->stream);
    g->off.release();
    g->adj.release();
    g->w.release();
    cudaStreamDestroy(g->stream);
    delete g;
    return PC_OK;
}

pc_status pc_graph_info(const pc_graph* g, uint64_t* n, uint64_t* m, int32_t* weighted) {
    clear_error();
    if (!g) return fail(PC_ERR_INVALID_INPUT, "null graph");
    if (n) *n = g->n;
    if (m) *m = g->m;
    if (weighted) *weighted = g->weighted ? 1 : 0;
    return PC_OK;
}

void* pc_graph_stream(const pc_graph* g) { return g ? (void*)g->stream : nullptr; }

pc_status pc_partition(pc_graph* g, const int32_t* v2p, pc_pgraph** out) {
    clear_error();
    if (!g || !out) return fail(PC_ERR_INVALID_INPUT, "null argument");
    *out = nullptr;
    PC_TRY(use_device(g));
    const uint64_t n = g->n;
    cudaStream_t s = g->stream;
    pc_pgraph* pg = new pc_pgraph();
    pg->g = g;
    pg->off = g->off.as<uint64_t>();
    pg->adj = g->adj.as<int32_t>();
    pg->w = g->weighted ? g->w.as<int32_t>() : nullptr;
    auto bail = [&](pc_status st) {
        const std::string msg = pc_last_error();
        cudaStreamSynchronize(s);
        if (pg->ev0) cudaEventDestroy(pg->ev0);
        if (pg->ev1) cudaEventDestroy(pg->ev1);
        delete pg;
        return fail(st, msg);
    };
    pc_status st;
    if ((st = pg->v2p.alloc(std::max<uint64_t>(n, 1) * 4, "vertex2partition")) != PC_OK) return bail(st);
    // checks, P = max + 1 (src/Graph.cpp:1021) and contiguity, on the device
    int32_t stats[3] = {0, 0, 0};
    if (v2p && n) {
        DevBuf dstat;
        if ((st = dstat.alloc(16, "partition checks")) != PC_OK) return bail(st);
        cudaError_t e = cudaMemcpyAsync(pg->v2p.p, v2p, n * 4, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(dstat.p, 0, 16, s);
        if (e != cudaSuccess) return bail(cuda_fail(e, "partition upload", __FILE__, __LINE__));
        k_v2p_stats<<<(unsigned)std::min<uint64_t>((uint64_t)sm_count(g->device) * 8, ceil_div(n, 256)), 256, 0, s>>>(
            pg->v2p.as<int32_t>(), n, dstat.as<int32_t>());
        count_launch();
        e = cudaMemcpyAsync(stats, dstat.p, 12, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return bail(cuda_fail(e, "partition checks", __FILE__, __LINE__));
        if (stats[0]) return bail(fail(PC_ERR_INVALID_INPUT, "partition ids must be non-negative"));
    } else if (n) {
        if (cudaMemsetAsync(pg->v2p.p, 0, n * 4, s) != cudaSuccess)
            return bail(fail(PC_ERR_CUDA, "memset of the partition vector failed"));
    }
    const int64_t P = (int64_t)stats[1] + 1;
    if (P > (1 << 24)) return bail(fail(PC_ERR_INVALID_INPUT, "more than 2^24 partitions"));
    const bool contiguous = stats[2] == 0;
    pg->P = (int32_t)P;
    pg->contiguous = contiguous;
    if ((st = pg->d_pstart.alloc((P + 1) * 8, "partition offsets")) != PC_OK) return bail(st);
    const unsigned nb = (unsigned)std::max<uint64_t>(1, ceil_div(n, 256));
    const unsigned ng = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sm_count(g->device) * 16,
                                                                           ceil_div(n + 1, 256)));
    // poffsets / plist (src/Graph.cpp:1024-1035): vertices per partition, ascending id
    if (contiguous) {
        k_partition_starts<<<ng, 256, 0, s>>>(pg->v2p.as<int32_t>(), n, P, pg->d_pstart.as<int64_t>());
        count_launch();
    } else {
        // plist = ids stably sorted by partition (an LSD radix sort is stable)
        if ((st = pg->new2old.alloc(n * 4, "new2old")) != PC_OK || (st = pg->old2new.alloc(n * 4, "old2new")) != PC_OK)
            return bail(st);
        DevBuf keys, ids, tmp;
        if ((st = keys.alloc(n * 4, "sort keys")) != PC_OK || (st = ids.alloc(n * 4, "sort values")) != PC_OK)
            return bail(st);
        int bits = 1;
        while ((1ll << bits) < P) ++bits;
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, pg->v2p.as<int32_t>(), keys.as<int32_t>(), ids.as<int32_t>(),
                                        pg->new2old.as<int32_t>(), (int64_t)n, 0, bits, s);
        if ((st = tmp.alloc(std::max<size_t>(tb, 256), "sort scratch")) != PC_OK) return bail(st);
        k_iota_i32<<<nb, 256, 0, s>>>(ids.as<int32_t>(), n);
        count_launch();
        cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp.p, tb, pg->v2p.as<int32_t>(), keys.as<int32_t>(),
                                                        ids.as<int32_t>(), pg->new2old.as<int32_t>(), (int64_t)n, 0,
                                                        bits, s);
        if (e != cudaSuccess) return bail(cuda_fail(e, "partition sort", __FILE__, __LINE__));
        count_launch();
        k_invert<<<nb, 256, 0, s>>>(pg->new2old.as<int32_t>(), n, pg->old2new.as<int32_t>());
        count_launch();
        k_partition_starts<<<ng, 256, 0, s>>>(keys.as<int32_t>(), n, P, pg->d_pstart.as<int64_t>());
        count_launch();
        e = cudaStreamSynchronize(s);  // keys, ids and tmp are released on return
        if (e != cudaSuccess) return bail(cuda_fail(e, "partition maps", __FILE__, __LINE__));
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return bail(cuda_fail(e, "kernel launch", __FILE__, __LINE__));
    pg->pstart.assign(P + 1, 0);
    e = cudaMemcpyAsync(pg->pstart.data(), pg->d_pstart.p, (P + 1) * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaEventCreate(&pg->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&pg->ev1);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return bail(cuda_fail(e, "partition offsets", __FILE__, __LINE__));
    g->live_views++;
    *out = pg;
    return PC_OK;
}

pc_status pc_pgraph_destroy(pc_pgraph* pg) {
    clear_error();
    if (!pg) return PC_OK;
    cudaSetDevice(pg->g->device);
    cudaStreamSynchronize(pg->g->stream);
    if (pg->ev0) cudaEventDestroy(pg->ev0);
    if (pg->ev1) cudaEventDestroy(pg->ev1);
    pg->g->live_views--;
    delete pg;
    return PC_OK;
}

pc_status pc_pgraph_info(const pc_pgraph* pg, uint64_t* n, uint64_t* m, int32_t* partitions) {
    clear_error();
    if (!pg) return fail(PC_ERR_INVALID_INPUT, "null partitioned graph");
    if (n) *n = pg->g->n;
    if (m) *m = pg->g->m;
    if (partitions) *partitions = pg->P;
    return PC_OK;
}

pc_status pc_pgraph_reorder(pc_pgraph* pg) {
    clear_error();
    if (!pg) return fail(PC_ERR_INVALID_INPUT, "null partitioned graph");
    pg->reordered_view = true;
    return PC_OK;
}

pc_status pc_pgraph_vertex_map(const pc_pgraph* pg, int32_t* old2new) {
    clear_error();
    if (!pg || !old2new) return fail(PC_ERR_INVALID_INPUT, "null argument");
    const uint64_t n = pg->g->n;
    if (api_is_internal(pg)) {
        for (uint64_t u = 0; u < n; ++u) old2new[u] = (int32_t)u;
        return PC_OK;
    }
    PC_TRY(use_device(pg->g));
    PC_CUDA(cudaMemcpy(old2new, pg->old2new.p, n * 4, cudaMemcpyDeviceToHost));
    return PC_OK;
}

pc_status pc_pgraph_layout(pc_pgraph* pg, uint64_t* vlist, int32_t* elist, int32_t* weights) {
    clear_error();
    if (!pg || !vlist || (pg->g->m && !elist)) return fail(PC_ERR_INVALID_INPUT, "null argument");
    PC_TRY(use_device(pg->g));
    const uint64_t n = pg->g->n, m = pg->g->m, PN = (uint64_t)pg->P * n;
    if (PN > (1ull << 31)) return fail(PC_ERR_INVALID_INPUT, "P*n too large for a materialised layout (limit 2^31)");
    if (n == 0) {
        vlist[0] = 0;
        return PC_OK;
    }
    const bool want_w = weights && pg->g->weighted;
    size_t temp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, (uint64_t*)nullptr, (uint64_t*)nullptr, (int64_t)(PN + 1));
    size_t need = (PN + 1) * 8 * 2 + temp_bytes + (m + 1) * 4 * 2;
    PC_TRY(scratch_reserve(pg, need));
    uint64_t* cnt = pg->scratch.take<uint64_t>(PN + 1);
    uint64_t* pos = pg->scratch.take<uint64_t>(PN + 1);
    void* tmp = pg->scratch.take<char>(temp_bytes);
    int32_t* oe = pg->scratch.take<int32_t>(m + 1);
    int32_t* ow = pg->scratch.take<int32_t>(m + 1);
    cudaStream_t s = pg->g->stream;
    PC_CUDA(cudaMemsetAsync(cnt, 0, (PN + 1) * 8, s));
    const int32_t* api2int = api_is_internal(pg) ? nullptr : pg->new2old.as<int32_t>();
    const int32_t* int2api = api_is_internal(pg) ? nullptr : pg->old2new.as<int32_t>();
    // With a reordered view, partitions are keyed by the original v2p of the
    // neighbour; rows are the API (new) ids.
    k_layout_count<<<(unsigned)ceil_div(n, 128), 128, 0, s>>>(pg->off, pg->adj, pg->v2p.as<int32_t>(), api2int, n, cnt);
    PC_LAUNCHED();
    PC_CUDA(cub::DeviceScan::ExclusiveSum(tmp, temp_bytes, cnt, pos, (int64_t)(PN + 1), s));
    count_launch();
    PC_CUDA(cudaMemcpyAsync(vlist, pos, (PN + 1) * 8, cudaMemcpyDeviceToHost, s));
    k_layout_fill<<<(unsigned)ceil_div(n, 128), 128, 0, s>>>(pg->off, pg->adj, pg->w, pg->v2p.as<int32_t>(), api2int,
                                                             int2api, n, pos, oe, want_w ? ow : nullptr);
    PC_LAUNCHED();
    if (m) PC_CUDA(cudaMemcpyAsync(elist, oe, m * 4, cudaMemcpyDeviceToHost, s));
    if (want_w && m) PC_CUDA(cudaMemcpyAsync(weights, ow, m * 4, cudaMemcpyDeviceToHost, s));
    return sync(pg);
}

pc_status pc_pgraph_evaluate(pc_pgraph* pg, int64_t* max_part_deg, int64_t* max_deg, double* balance_ratio) {
    clear_error();
    if (!pg) return fail(PC_ERR_INVALID_INPUT, "null partitioned graph");
    PC_TRY(use_device(pg->g));
    const uint64_t n = pg->g->n, m = pg->g->m;
    std::vector<uint64_t> off(n + 1);
    std::vector<int32_t> adj(m), v2p(n);
    PC_CUDA(cudaMemcpy(off.data(), pg->off, (n + 1) * 8, cudaMemcpyDeviceToHost));
    if (m) PC_CUDA(cudaMemcpy(adj.data(), pg->adj, m * 4, cudaMemcpyDeviceToHost));
    if (n) PC_CUDA(cudaMemcpy(v2p.data(), pg->v2p.p, n * 4, cudaMemcpyDeviceToHost));
    int64_t mpd = 0, md = 0;
    std::vector<int64_t> c(pg->P, 0);
    for (uint64_t u = 0; u < n; ++u) {
        for (uint64_t e = off[u]; e < off[u + 1]; ++e) c[v2p[adj[e]]]++;
        for (uint64_t e = off[u]; e < off[u + 1]; ++e) {
            int32_t k = v2p[adj[e]];
            if (c[k] > mpd) mpd = c[k];
            c[k] = 0;
        }
        md = std::max<int64_t>(md, (int64_t)(off[u + 1] - off[u]));
    }
    if (max_part_deg) *max_part_deg = mpd;
    if (max_deg) *max_deg = md;
    // src/Graph.cpp:1471: (P * max_part_deg) / max_deg
    if (balance_ratio) *balance_ratio = md ? (double)((int64_t)pg->P * mpd) / (double)md : 0.0;
    return PC_OK;
}

}  // extern "C"
