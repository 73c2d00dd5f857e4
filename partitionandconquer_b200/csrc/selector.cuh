// Per-partition kernel selection for the intersection kernels: unit
// features, the plain autotuned heuristic and the learned (MLP) selector.
#pragma once
#include <stdint.h>

#include <vector>

#include "pc_internal.cuh"

namespace pc {

// Raw per-unit statistics gathered on the device (k_unit_stats):
// 0 pivots, 1 in-edges, 2 sum |N+(b)|, 3 max |N+(b)|, 4 max pivot id + 1,
// 5 sum over in-edges (c->b) of |N+(c)|, 6 sum log2(1+deg)*1024,
// 7 sum log2(1+deg)^2*1024, 8 in-edges whose |N+(c)| >= 32.
constexpr int kRawStats = 9;
// Raw features (floats) kept per unit: the 9 statistics above with the log
// moments turned into mean/variance, plus 9 = in-edges per pivot.
constexpr int kNumFeatures = 10;
// Model input width (derived, standardised features).
constexpr int kMlpIn = 12;
constexpr int kMlpHidden = 64;
constexpr int kMlpOut = PC_NUM_VARIANTS;
constexpr int kMlpParams = kMlpIn * kMlpHidden + kMlpHidden + kMlpHidden * kMlpHidden + kMlpHidden +
                           kMlpHidden * kMlpOut + kMlpOut;

void raw_to_features(const unsigned long long* raw, float* f);
inline double feat_raw_scan(const float* f) { return f[5]; }
// Model inputs (before standardisation) from raw features.
void features_to_inputs(const float* f, float* x);

struct HeuristicParams {
    // Defaults: the thresholds pc_selector_autotune chose from in-situ unit
    // costs of RMAT graphs at scales 20, 22 and 24 (with ER and Chung-Lu).
    double min_in_per_pivot_cta = 128.0;  // in-edges per pivot to use a bitmap form
    double warp_scan = 256.0;             // mean prefix bound for 32 lanes per in-neighbour
    double group_scan = 0.0;              // ... for 8 lanes per in-neighbour
    double matrix_scan = 256.0;           // ... for the in-neighbour-major hub form (ids < 2^16)
};
HeuristicParams heuristic_params();
void set_heuristic_params(const HeuristicParams& hp);

namespace tc {
int heuristic_choice(const float* f, const HeuristicParams& hp);
bool variant_feasible(int v, const float* f);
}  // namespace tc

// Learned selector state (process-wide).  The version changes whenever the
// model or the heuristic thresholds change (plans are cached per version).
bool selector_ready(int device);
uint64_t selector_version();
// Learned choices for all units (batched GPU inference), each judged against
// the heuristic; units without work get -1.
pc_status selector_choose_batch(const std::vector<float>& feat, size_t U, std::vector<int8_t>* choice);

// TC planner hooks used by the selector (tc.cu).
pc_status tc_count(pc_pgraph* pg, int32_t variant, uint64_t* count, pc_tc_stats* stats);
pc_status tc_time_unit(pc_pgraph* pg, size_t unit, int variant, double* ms, uint64_t* count);
pc_status tc_profile_variant(pc_pgraph* pg, int variant, std::vector<double>* unit_ms, uint64_t* count);
pc_status tc_vertex_triangles(pc_pgraph* pg, int32_t variant, unsigned long long* d_tri, uint64_t* count);
pc_status tc_edge_triangles(pc_pgraph* pg, int32_t variant, uint32_t* d_ecnt, uint64_t* count);
pc_status tc_assign(pc_pgraph* pg, int32_t variant, const std::vector<float>& feat, size_t U,
                    std::vector<int8_t>* assign, int* selector_used);
pc_status tc_ensure_features(pc_pgraph* pg);

}  // namespace pc
