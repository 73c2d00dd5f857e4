// Counter-based random numbers for the seeded synthetic graphs.
//
// Every random draw is a pure function of (graph key, counter), so the host
// generator (OpenMP) and the device generator (CUDA) produce bit-identical
// edge lists, whatever the thread count or launch shape.
//
// The mixing function is the SplitMix64 output function (G. Steele, D. Lea,
// C. Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014):
// draw(c) = mix(key + c * golden_gamma).  The RMAT quadrant rule is the one of
// Chakrabarti, Zhan, Faloutsos, "R-MAT: A recursive model for graph mining"
// (SDM 2004) with probabilities compared as 32-bit fixed-point thresholds, so
// no floating point enters the edge stream.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define PC_HD __host__ __device__ __forceinline__
#else
#define PC_HD static inline
#endif

#define PC_GOLDEN_GAMMA 0x9E3779B97F4A7C15ULL

PC_HD uint64_t pc_mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// Per-graph key: separates streams of different seeds and generator kinds.
PC_HD uint64_t pc_graph_key(uint64_t seed, uint64_t kind) {
    return pc_mix64(pc_mix64(seed * PC_GOLDEN_GAMMA + 0x632BE59BD9B4E019ULL) ^ (kind * 0xD1B54A32D192ED03ULL));
}

PC_HD uint64_t pc_draw(uint64_t key, uint64_t counter) {
    return pc_mix64(key + counter * PC_GOLDEN_GAMMA);
}

enum { PC_GEN_RMAT = 1, PC_GEN_ER = 2, PC_GEN_CHUNG_LU = 3, PC_GEN_WEIGHT = 4, PC_GEN_PRIORITY = 5, PC_GEN_BATCH = 6,
       PC_GEN_PARTITION = 7 };

// RMAT quadrant thresholds for (a, b, c, d) = (0.57, 0.19, 0.19, 0.05):
// r < A -> (0,0); A <= r < AB -> column bit; AB <= r < ABC -> row bit; else both.
#define PC_RMAT_A   2448131358u   /* floor(0.57 * 2^32) */
#define PC_RMAT_AB  3264175144u   /* floor(0.76 * 2^32) */
#define PC_RMAT_ABC 4080218931u   /* floor(0.95 * 2^32) */

// Edge k of an RMAT graph of 2^scale vertices.  Two 32-bit quadrant draws come
// from each 64-bit output; level l decides bit (scale-1-l) of both endpoints.
PC_HD void pc_rmat_edge(uint64_t key, uint64_t k, uint32_t scale, uint32_t* u, uint32_t* v) {
    uint32_t uu = 0, vv = 0;
    for (uint32_t l = 0; l < scale; l += 2) {
        uint64_t x = pc_draw(key, (k << 5) | (l >> 1));
        for (uint32_t h = 0; h < 2 && l + h < scale; ++h) {
            uint32_t r = (uint32_t)(x >> (32 * h));
            uint32_t bit = 1u << (scale - 1 - (l + h));
            if (r >= PC_RMAT_ABC) { uu |= bit; vv |= bit; }
            else if (r >= PC_RMAT_AB) { uu |= bit; }
            else if (r >= PC_RMAT_A) { vv |= bit; }
        }
    }
    *u = uu;
    *v = vv;
}

// Edge k of an Erdos-Renyi G(n = 2^scale, m) multigraph draw (uniform endpoints).
PC_HD void pc_er_edge(uint64_t key, uint64_t k, uint32_t scale, uint32_t* u, uint32_t* v) {
    uint64_t x = pc_draw(key, k);
    *u = (uint32_t)(x >> (64 - scale));
    *v = (uint32_t)((x & 0xFFFFFFFFull) >> (32 - scale));
}

// Symmetric integer edge weight in [1, wmax] from the unordered pair {a, b}.
PC_HD int32_t pc_edge_weight(uint64_t key, uint32_t a, uint32_t b, int32_t wmax) {
    uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    uint64_t x = pc_draw(key, ((uint64_t)lo << 32) | hi);
    return 1 + (int32_t)(((x >> 32) * (uint64_t)wmax) >> 32);
}

// Seed-hashed vertex priority for the MIS order: the top 33 bits of
// draw(key, v) above the 31-bit id, so priorities are distinct and ties can
// never occur.
PC_HD uint64_t pc_vertex_priority(uint64_t key, uint32_t v) {
    return ((pc_draw(key, v) >> 31) << 31) | (uint64_t)(v & 0x7FFFFFFFu);
}
