// Internal definitions shared by the CUDA translation units of libpc.so.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/pc.h"

namespace pc {

// ---- errors --------------------------------------------------------------

void set_error(const std::string& msg);
void clear_error();
pc_status fail(pc_status st, const std::string& msg);
pc_status cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define PC_CUDA(call)                                                   \
    do {                                                                \
        cudaError_t _e = (call);                                        \
        if (_e != cudaSuccess) return pc::cuda_fail(_e, #call, __FILE__, __LINE__); \
    } while (0)

#define PC_TRY(call)                    \
    do {                                \
        pc_status _s = (call);          \
        if (_s != PC_OK) return _s;     \
    } while (0)

// Checks the launch that was just issued.
#define PC_LAUNCHED()                                                   \
    do {                                                                \
        pc::count_launch();                                             \
        cudaError_t _e = cudaGetLastError();                            \
        if (_e != cudaSuccess) return pc::cuda_fail(_e, "kernel launch", __FILE__, __LINE__); \
    } while (0)

void count_launch();

// ---- device memory -------------------------------------------------------

// Owning device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int dev = 0;  // device whose pool holds the block
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    pc_status alloc(size_t nbytes, const char* what);
    pc_status ensure(size_t nbytes, const char* what);  // grow-only
    void release();
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

// Bump allocator over one grow-only buffer; reset at the start of each call.
struct Scratch {
    DevBuf buf;
    size_t used = 0;
    size_t high = 0;  // bytes requested by the largest call so far
    std::vector<size_t> pending;
    void reset() { used = 0; }
    // Plan-then-allocate: callers request every region first with take(),
    // which only succeeds when capacity is enough; grow() is used on miss.
    template <class T>
    T* take(size_t count) {
        size_t off = (used + 255) & ~(size_t)255;
        size_t need = off + count * sizeof(T);
        if (need > buf.bytes) return nullptr;
        used = need;
        if (used > high) high = used;
        return reinterpret_cast<T*>(reinterpret_cast<char*>(buf.p) + off);
    }
};

// ---- handles -------------------------------------------------------------

}  // namespace pc

struct pc_graph {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint64_t n = 0, m = 0;
    bool weighted = false;
    pc::DevBuf off;   // uint64 [n+1]
    pc::DevBuf adj;   // int32  [m + pad]
    pc::DevBuf w;     // int32  [m] or empty
    int live_views = 0;
};

struct pc_pgraph {
    pc_graph* g = nullptr;
    int32_t P = 1;
    bool contiguous = true;      // internal ids == original ids
    bool reordered_view = false; // API ids are the internal ids
    // internal (partition-contiguous) CSR; aliases g when contiguous
    uint64_t* off = nullptr;
    int32_t* adj = nullptr;
    int32_t* w = nullptr;
    pc::DevBuf old2new, new2old;  // int32 [n] when !contiguous
    pc::DevBuf v2p;               // int32 [n], original ids
    std::vector<int64_t> pstart;  // P+1 partition boundaries (internal ids)
    pc::DevBuf d_pstart;          // int64 [P+1]
    pc::DevBuf dplus;             // uint32 [n]: |N(u) & [0,u)| (internal ids)
    pc::DevBuf unit_of;           // int32 [n]: planning unit of each vertex (tc.cu)
    pc::Scratch scratch;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // planner state (tc.cu)
    std::vector<float> part_features;  // per-unit features (lazy)
    std::vector<int64_t> unit_lo, unit_hi;  // planning units (plist position ranges)
    bool features_ready = false;
    uint64_t plan_key = 0;                  // selector version of the cached plan
    std::vector<int8_t> plan_assign;        // cached variant per unit
};

namespace pc {

inline uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

// Number of SMs of the handle's device (cached per device).
int sm_count(int device);

// Sets the handle's device current.
pc_status use_device(const pc_graph* g);

// Ensures the scratch arena of pg holds `bytes`; resets it.
pc_status scratch_reserve(pc_pgraph* pg, size_t bytes);

// Copies a host array into a scratch region.
template <class T>
pc_status upload(pc_pgraph* pg, const T* host, size_t count, T** dev) {
    *dev = pg->scratch.take<T>(count);
    if (!*dev) return fail(PC_ERR_OOM, "scratch arena too small (internal sizing error)");
    if (count) PC_CUDA(cudaMemcpyAsync(*dev, host, count * sizeof(T), cudaMemcpyHostToDevice, pg->g->stream));
    return PC_OK;
}

// Maps API vertex ids to internal ids in place on the device (no-op when the
// internal id space is the API id space).
pc_status map_ids_to_internal(pc_pgraph* pg, int32_t* d_ids, uint64_t count);
// Writes out_api[i] = in_internal[internal id of API vertex i] (a gather by old2new).
pc_status gather_to_api_i32(pc_pgraph* pg, const int32_t* in_internal, int32_t* out_api);
pc_status gather_to_api_f32(pc_pgraph* pg, const float* in_internal, float* out_api);
pc_status gather_to_api_f64(pc_pgraph* pg, const double* in_internal, double* out_api);
bool api_is_internal(const pc_pgraph* pg);
// out_internal[u] = in_api[API id of u] (a gather by old2new).
pc_status gather_to_internal_i32(pc_pgraph* pg, const int32_t* in_api, int32_t* out_internal);
pc_status gather_to_internal_f32(pc_pgraph* pg, const float* in_api, float* out_internal);
pc_status gather_to_internal_f64(pc_pgraph* pg, const double* in_api, double* out_internal);
// Internal id of one API vertex id (synchronous).
int32_t to_internal_id(const pc_pgraph* pg, int32_t api_id);

// Lazily computes pg->dplus.
pc_status ensure_dplus(pc_pgraph* pg);

// Synchronises the handle's stream and converts a device error to a status.
pc_status sync(pc_pgraph* pg);

}  // namespace pc
