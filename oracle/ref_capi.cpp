// TEST INFRASTRUCTURE -- a C entry layer over the UNMODIFIED reference
// (src/Graph.cpp + src/Graph.hpp of PartitionAndConquer), compiled together
// with it by oracle/Makefile into oracle/_ref/libpcref.so.  Used by the tests
// to pin the oracle and by bench.py's reference arm to time the reference's
// own OpenMP code.  Nothing here re-implements an algorithm: every function
// calls the reference member named beside it.
//
// The layout members of Partitioned_Graph are private in the reference; this
// translation unit reads them (for the layout parity test) by compiling the
// class declaration with `private` mapped to `public`, which changes access
// only, not the class layout.
// Every header Graph.hpp pulls in is included first, so the access remapping
// below touches the reference's class declarations only.
#include <omp.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <boost/dynamic_bitset.hpp>
#include <cassert>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iostream>
#include <numeric>
#include <queue>
#include <random>
#include <string>
#include <unordered_set>
#include <utility>
#include <vector>

#define private public
#include "Graph.hpp"
#undef private

extern "C" {

// Graph::Graph(csrdir, is_weighted) (src/Graph.cpp:92-137).
void* ref_graph_load(const char* dir, int weighted) { return new Graph(std::string(dir), weighted != 0); }
void ref_graph_free(void* g) { delete static_cast<Graph*>(g); }
uint64_t ref_graph_n(void* g) { return static_cast<Graph*>(g)->get_vertex_num(); }
uint64_t ref_graph_m(void* g) { return static_cast<Graph*>(g)->get_edge_num(); }

// Partitioned_Graph::Partitioned_Graph (src/Graph.cpp:1017-1069).
void* ref_pgraph_new(void* g, const int32_t* v2p, uint64_t n, int threads) {
    std::vector<int> p(v2p, v2p + n);
    return new Partitioned_Graph(*static_cast<Graph*>(g), p, threads);
}
void ref_pgraph_free(void* pg) { delete static_cast<Partitioned_Graph*>(pg); }
uint64_t ref_pgraph_partitions(void* pg) { return static_cast<Partitioned_Graph*>(pg)->get_partition_num(); }
// Partitioned_Graph::reorder (src/Graph.cpp:1665-1699).
void ref_pgraph_reorder(void* pg) { static_cast<Partitioned_Graph*>(pg)->reorder(); }
// Layout members (src/Graph.hpp:149-151): csr_vlist (P*n+1), csr_elist, csr_weight.
void ref_pgraph_layout(void* pg, uint64_t* vlist, int32_t* elist, int32_t* weights) {
    auto* p = static_cast<Partitioned_Graph*>(pg);
    std::memcpy(vlist, p->csr_vlist.data(), p->csr_vlist.size() * sizeof(uint64_t));
    std::memcpy(elist, p->csr_elist.data(), p->csr_elist.size() * sizeof(int32_t));
    if (weights && !p->csr_weight.empty())
        std::memcpy(weights, p->csr_weight.data(), p->csr_weight.size() * sizeof(int32_t));
}
// Partitioned_Graph::evaluate_partition (src/Graph.cpp:1460-1473) prints its figures.
void ref_pgraph_evaluate(void* pg) { static_cast<Partitioned_Graph*>(pg)->evaluate_partition(); }

// Triangle counting: Graph::solve_triangle_counting_{merge,galloping}
// (src/Graph.cpp:342-368) and Partitioned_Graph::... (src/Graph.cpp:1326-1362).
uint64_t ref_tc_graph(void* g, int galloping, int threads) {
    auto* G = static_cast<Graph*>(g);
    return galloping ? G->solve_triangle_counting_galloping(threads) : G->solve_triangle_counting_merge(threads);
}
uint64_t ref_tc_pgraph(void* pg, int galloping) {
    auto* G = static_cast<Partitioned_Graph*>(pg);
    return galloping ? G->solve_triangle_counting_galloping() : G->solve_triangle_counting_merge();
}
// One oriented edge (u, v), v < u: Graph::cnt_common_neis_less_than_merge
// (src/Graph.cpp:272-285), the body of the TC loop (src/Graph.cpp:358-365).
uint64_t ref_tc_rows(void* g, const int32_t* rows, uint64_t nrows, int threads) {
    auto* G = static_cast<Graph*>(g);
    const EID* vl = G->get_csr_vlist();
    const VID* el = G->get_csr_elist();
    size_t res = 0;
    // the reference loop's own schedule: `omp parallel for` without a
    // schedule clause (static) over the rows, as Graph::solve_triangle_counting_merge
#pragma omp parallel for num_threads(threads) schedule(static) reduction(+ : res)
    for (int64_t i = 0; i < (int64_t)nrows; ++i) {
        VID u = rows[i];
        for (EID j = vl[u]; j < vl[u + 1]; ++j) {
            VID v = el[j];
            if (u <= v) continue;
            res += G->cnt_common_neis_less_than_merge(u, v, v);
        }
    }
    return res;
}

// LCC: Graph::solve_lcc_{merge,galloping} (src/Graph.cpp:814-840),
// Partitioned_Graph::solve_lcc_* (src/Graph.cpp:2197-2261).
void ref_lcc_graph(void* g, int galloping, int threads, double* out) {
    std::vector<double> r;
    auto* G = static_cast<Graph*>(g);
    if (galloping) G->solve_lcc_galloping(r, threads); else G->solve_lcc_merge(r, threads);
    std::memcpy(out, r.data(), r.size() * sizeof(double));
}
void ref_lcc_pgraph(void* pg, int galloping, double* out) {
    std::vector<double> r;
    auto* G = static_cast<Partitioned_Graph*>(pg);
    if (galloping) G->solve_lcc_galloping(r); else G->solve_lcc_merge(r);
    std::memcpy(out, r.data(), r.size() * sizeof(double));
}

// Jaccard over a query list: Graph::solve_jsim_merge (src/Graph.cpp:798-812)
// and, for the record, Partitioned_Graph::solve_jsim_merge (src/Graph.cpp:2162-2195).
void ref_jsim_graph(void* g, const int32_t* q, int32_t nq, int threads, double* out) {
    std::vector<VID> qs(q, q + nq);
    std::vector<double> r;
    static_cast<Graph*>(g)->solve_jsim_merge(qs, r, threads);
    std::memcpy(out, r.data(), r.size() * sizeof(double));
}
void ref_jsim_pgraph(void* pg, const int32_t* q, int32_t nq, double* out) {
    std::vector<VID> qs(q, q + nq);
    std::vector<double> r;
    static_cast<Partitioned_Graph*>(pg)->solve_jsim_merge(qs, r);
    std::memcpy(out, r.data(), r.size() * sizeof(double));
}

// Batched pair counts: Graph::batch_cnt_common_neis_merge (src/Graph.cpp:431-438),
// Partitioned_Graph::batch_cnt_common_neis_merge (src/Graph.cpp:1421-1432).
void ref_batch_pairs(void* obj, int partitioned, const int32_t* pairs, uint64_t nq, int threads, uint64_t* out) {
    std::vector<std::pair<VID, VID>> qs(nq);
    for (uint64_t i = 0; i < nq; ++i) qs[i] = {pairs[2 * i], pairs[2 * i + 1]};
    std::vector<size_t> r(nq, 0);
    if (partitioned) static_cast<Partitioned_Graph*>(obj)->batch_cnt_common_neis_merge(qs, r);
    else static_cast<Graph*>(obj)->batch_cnt_common_neis_merge(qs, r, threads);
    for (uint64_t i = 0; i < nq; ++i) out[i] = r[i];
}
// k-sets: src/Graph.cpp:440-447 and 1434-1445.
void ref_batch_sets(void* obj, int partitioned, const int32_t* ids, const uint64_t* offs, uint64_t nq, int threads,
                    uint64_t* out) {
    std::vector<std::vector<VID>> qs(nq);
    for (uint64_t i = 0; i < nq; ++i) qs[i].assign(ids + offs[i], ids + offs[i + 1]);
    std::vector<size_t> r(nq, 0);
    if (partitioned) static_cast<Partitioned_Graph*>(obj)->batch_cnt_common_neis_merge(qs, r);
    else static_cast<Graph*>(obj)->batch_cnt_common_neis_merge(qs, r, threads);
    for (uint64_t i = 0; i < nq; ++i) out[i] = r[i];
}

// BFS parents: Graph::solve_bfs (src/Graph.cpp:621-646).  (The partitioned
// BFS, src/Graph.cpp:1701-1762, does not terminate on these graphs and is not
// called.)
void ref_bfs_graph(void* g, int32_t src, int32_t* parents) {
    std::vector<VID> p;
    static_cast<Graph*>(g)->solve_bfs(src, p);
    std::memcpy(parents, p.data(), p.size() * sizeof(int32_t));
}

// SSSP: Graph::solve_sssp (src/Graph.cpp:842-868), Partitioned_Graph::solve_sssp
// (src/Graph.cpp:2263-2309) with dist pre-filled as in src/test.cpp:202-203.
void ref_sssp(void* obj, int partitioned, uint64_t n, int32_t src, int32_t* out) {
    std::vector<int> d(n, INT_MAX / 2);
    if (partitioned) static_cast<Partitioned_Graph*>(obj)->solve_sssp(src, d);
    else static_cast<Graph*>(obj)->solve_sssp(d, src);
    std::memcpy(out, d.data(), n * sizeof(int32_t));
}

// PageRank: Partitioned_Graph::page_rank (src/Graph.cpp:1555-1602) and
// Graph::page_rank (src/Graph.cpp:534-554); init as src/test.cpp:270.
void ref_pagerank(void* obj, int partitioned, uint64_t n, float damping, int iters, int threads, float* out) {
    std::vector<float> pr(n, 1.0f);
    if (partitioned) static_cast<Partitioned_Graph*>(obj)->page_rank(pr, damping, iters);
    else static_cast<Graph*>(obj)->page_rank(pr, damping, iters, threads);
    std::memcpy(out, pr.data(), n * sizeof(float));
}

// k-core: Graph::solve_kcore (src/Graph.cpp:662-719), Partitioned_Graph::solve_kcore
// (src/Graph.cpp:1863-1942).
void ref_kcore(void* obj, int partitioned, uint64_t n, int threads, int32_t* out) {
    std::vector<int> c(n, 0);
    if (partitioned) static_cast<Partitioned_Graph*>(obj)->solve_kcore(c);
    else static_cast<Graph*>(obj)->solve_kcore(c, threads);
    std::memcpy(out, c.data(), n * sizeof(int32_t));
}

// MIS: Graph::solve_mis (src/Graph.cpp:721-780), Partitioned_Graph::solve_mis
// (src/Graph.cpp:1944-2044).
void ref_mis(void* obj, int partitioned, uint64_t n, int threads, int32_t* out) {
    std::vector<int> r(n, 0);
    if (partitioned) static_cast<Partitioned_Graph*>(obj)->solve_mis(r);
    else static_cast<Graph*>(obj)->solve_mis(r, threads);
    std::memcpy(out, r.data(), n * sizeof(int32_t));
}

// CDLP: Graph::solve_cdlp (src/Graph.cpp:648-660), Partitioned_Graph::solve_cdlp
// (src/Graph.cpp:1843-1861); labels in/out.
void ref_cdlp(void* obj, int partitioned, uint64_t n, int iters, int threads, int32_t* labels) {
    std::vector<int> l(labels, labels + n);
    if (partitioned) static_cast<Partitioned_Graph*>(obj)->solve_cdlp(l, iters);
    else static_cast<Graph*>(obj)->solve_cdlp(l, iters, threads);
    std::memcpy(labels, l.data(), n * sizeof(int32_t));
}

// Friend triangles: Graph::solve_friend_triangle_{merge,galloping}
// (src/Graph.cpp:309-340), Partitioned_Graph:: forms (src/Graph.cpp:1222-1264).
uint64_t ref_friend_triangle(void* obj, int partitioned, int galloping, int32_t root, const int32_t* nodes,
                             uint64_t nn, int threads) {
    std::vector<VID> q(nodes, nodes + nn);
    if (partitioned) {
        auto* p = static_cast<Partitioned_Graph*>(obj);
        return galloping ? p->solve_friend_triangle_galloping(root, q) : p->solve_friend_triangle_merge(root, q);
    }
    auto* g = static_cast<Graph*>(obj);
    return galloping ? g->solve_friend_triangle_galloping(root, q, threads)
                     : g->solve_friend_triangle_merge(root, q, threads);
}

// Partitioned_Graph::solve_square_counting (src/Graph.cpp:1291-1324).
uint64_t ref_square_count(void* pg) { return static_cast<Partitioned_Graph*>(pg)->solve_square_counting(); }

}  // extern "C"
