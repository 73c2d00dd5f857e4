// Grid-wide barrier for persistent kernels started with a cooperative launch
// (every CTA of the grid is resident, so every CTA can reach the barrier).
//
// Every wait is bounded by a wall-clock limit read from %globaltimer: a CTA
// that waits longer, or that sees another CTA's error, records the error and
// the barrier returns false, so the kernel can return and the host can read
// the status instead of the GPU spinning for ever.
#pragma once
#include <cstdint>

namespace pc {

struct GridBarrier {
    unsigned count;  // CTAs arrived in the current generation
    unsigned gen;    // generation, bumped by the last CTA to arrive
    int err;         // 1: a wait ran out of time; 2: a step bound was hit
    int pad;
};

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// All threads of every CTA call it.  Writes made before it (plain stores and
// atomics) are visible to every CTA after it, to loads that bypass L1
// (__ldcg) or to atomics.
__device__ __forceinline__ bool grid_sync(GridBarrier* gb, uint64_t limit_ns) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        // the generation is read before arriving: the last CTA can only bump
        // it after this CTA's arrival
        const unsigned g = ld_acquire_u32(&gb->gen);
        __threadfence();
        const unsigned arrived = atomicAdd(&gb->count, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(&gb->count, 0u);
            __threadfence();
            atomicAdd(&gb->gen, 1u);
        } else {
            const uint64_t t0 = global_ns();
            for (;;) {
                if (ld_acquire_u32(&gb->gen) != g) break;
                if (*(volatile int*)&gb->err) { ok = 0; break; }
                if (global_ns() - t0 > limit_ns) {
                    atomicExch(&gb->err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace pc
