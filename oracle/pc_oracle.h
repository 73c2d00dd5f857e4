/* TEST INFRASTRUCTURE -- declarations of the CPU oracle (see pc_oracle.c). */
#ifndef PC_ORACLE_H
#define PC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

uint64_t or_tc_merge(uint64_t n, const uint64_t* vl, const int32_t* el);
uint64_t or_friend_triangle(uint64_t n, const uint64_t* vl, const int32_t* el, int32_t root, const int32_t* nodes,
                            uint64_t nn);
uint64_t or_square_count(uint64_t n, const uint64_t* vl, const int32_t* el);
uint64_t or_tc_galloping(uint64_t n, const uint64_t* vl, const int32_t* el);
uint64_t or_tc_rows(uint64_t n, const uint64_t* vl, const int32_t* el, const int32_t* rows, uint64_t nrows);
int or_layout(uint64_t n, const uint64_t* vl, const int32_t* el, const int32_t* w, const int32_t* v2p, int32_t P,
              uint64_t* out_vl, int32_t* out_el, int32_t* out_w);
uint64_t or_tc_partitioned(uint64_t n, const uint64_t* pvl, const int32_t* pel, int32_t P);
void or_lcc(uint64_t n, const uint64_t* vl, const int32_t* el, double* out);
void or_jaccard_edges(uint64_t n, const uint64_t* vl, const int32_t* el, float* out);
void or_jaccard_rows(uint64_t n, const uint64_t* vl, const int32_t* el, const int32_t* rows, uint64_t nrows,
                     float* out);
void or_jaccard_audit(uint64_t n, const uint64_t* vl, const int32_t* el, const float* J, uint64_t* sum_c,
                      uint64_t* bad_roundtrip, uint64_t* bad_twin);
void or_jaccard_queries(uint64_t n, const uint64_t* vl, const int32_t* el, const int32_t* q, int32_t nq, double* out);
void or_batch_pairs(uint64_t n, const uint64_t* vl, const int32_t* el, const int32_t* pairs, uint64_t nq, uint64_t* out);
void or_batch_sets(uint64_t n, const uint64_t* vl, const int32_t* el, const int32_t* ids, const uint64_t* offs,
                   uint64_t nq, uint64_t* out);
void or_bfs(uint64_t n, const uint64_t* vl, const int32_t* el, int32_t src, int32_t* rank);
void or_sssp(uint64_t n, const uint64_t* vl, const int32_t* el, const int32_t* w, int32_t src, int32_t* dist);
void or_pagerank_f64(uint64_t n, const uint64_t* vl, const int32_t* el, double damping, int32_t iters,
                     const double* init, double* out);
void or_mis_priority(uint64_t n, const uint64_t* vl, const int32_t* el, const uint64_t* priority, int32_t* res);
int32_t or_kcore(uint64_t n, const uint64_t* vl, const int32_t* el, int32_t* core);
void or_mis(uint64_t n, const uint64_t* vl, const int32_t* el, int32_t* res);
void or_cdlp(uint64_t n, const uint64_t* vl, const int32_t* el, int32_t iters, int32_t* labels);

#ifdef __cplusplus
}
#endif
#endif
