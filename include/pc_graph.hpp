// pc_graph.hpp -- C++ host classes with the reference's API (src/Graph.hpp of
// PartitionAndConquer): class Graph and class Partitioned_Graph, same method
// names, argument meaning and result vectors.  Loading, preprocessing and
// partitioning run on the host; every algorithm forwards to the C ABI of
// libpc.so (pc.h), which runs it on the GPU.  There is no CPU fallback: a
// failed call throws pc::Error carrying the pc_status and message.
#pragma once
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "pc.h"

namespace pc {

typedef int VID;                 // src/Graph.hpp:23
typedef unsigned long long EID;  // src/Graph.hpp:24
typedef int Weight;              // src/Graph.hpp:25

class Error : public std::runtime_error {
   public:
    Error(pc_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
    pc_status status;
};

class Partitioned_Graph;

class Graph {
   public:
    // Text edge list: '#'/'%' comment lines, "u v" per line, self-loops
    // dropped, symmetrised, sorted, de-duplicated; ids shifted down by one
    // unless a 0 id appears (src/Graph.cpp:27-90).
    explicit Graph(const std::string graphfile);
    // The same text loader with the adjacency build (symmetrise, sort,
    // deduplicate) done on the GPU by pc_graph_from_edges; identical arrays.
    struct OnDevice {};
    Graph(const std::string graphfile, OnDevice);
    // Binary CSR directory: csr_vlist.bin / csr_elist.bin / csr_weight.bin
    // (src/Graph.cpp:92-137).  Throws on a missing or malformed file.
    Graph(const std::string csrdir, bool is_weighted);
    explicit Graph(const std::vector<std::vector<VID>>& adj_list);
    Graph(std::vector<EID> vlist, std::vector<VID> elist, std::vector<Weight> weights = {});
    ~Graph();
    Graph(const Graph&) = delete;
    Graph& operator=(const Graph&) = delete;

    // accessors (src/Graph.cpp:151-307)
    const EID* get_csr_vlist() const { return csr_vlist.data(); }
    const VID* get_csr_elist() const { return csr_elist.data(); }
    const Weight* get_csr_weight() const { return csr_weight.data(); }
    bool has_edge(VID u, VID v) const;
    bool has_directed_edge(VID u, VID v) const;
    bool is_weighted() const { return !csr_weight.empty(); }
    EID get_edge_num() const { return edge_num; }
    VID get_vertex_num() const { return (VID)vertex_num; }
    size_t get_deg(VID u) const { return csr_vlist[u + 1] - csr_vlist[u]; }
    size_t get_max_deg() const;
    void get_degs(std::vector<int>& degs) const;
    void get_neis(VID u, std::vector<VID>& neis) const;

    // files (src/Graph.cpp:595-605) and the preprocess tool's weights
    // (src/preprocess.cpp:10-37: rand() % floor(log2 n) + 1, symmetric)
    void save_as_csr_binfile(const std::string csr_vlist_binfile, const std::string csr_elist_binfile);
    void add_reference_weights();
    void save_weight_binfile(const std::string csr_weight_binfile) const;

    // partitioners (host; src/Graph.cpp:564-570, 898-967)
    void random_partition(const size_t partition_num, std::vector<int>& vertex2partition);
    // greedy_partition seeds its shuffles from `seed` instead of random_device.
    void greedy_partition(const size_t partition_number, std::vector<int>& vertex2partition, uint64_t seed = 1);

    // algorithms on the GPU (unpartitioned forms; num_threads is accepted and ignored)
    size_t solve_triangle_counting_galloping(const int num_threads) const;
    size_t solve_triangle_counting_merge(const int num_threads) const;
    // src/Graph.cpp:309-340
    size_t solve_friend_triangle_galloping(const VID root, const std::vector<VID>& nodes, const int num_threads) const;
    size_t solve_friend_triangle_merge(const VID root, const std::vector<VID>& nodes, const int num_threads) const;
    void batch_cnt_common_neis_merge(const std::vector<std::pair<VID, VID>>& queries, std::vector<size_t>& res,
                                     int num_threads) const;
    void batch_cnt_common_neis_merge(const std::vector<std::vector<VID>>& queries, std::vector<size_t>& res,
                                     int num_threads) const;
    void batch_cnt_common_neis_galloping(const std::vector<std::pair<VID, VID>>& queries, std::vector<size_t>& res,
                                         int num_threads) const;
    void solve_jsim_merge(const std::vector<VID>& queries, std::vector<double>& res, int num_threads) const;
    void solve_jsim_galloping(const std::vector<VID>& queries, std::vector<double>& res, int num_threads) const;
    void solve_lcc_merge(std::vector<double>& res, int num_threads) const;
    void solve_lcc_galloping(std::vector<double>& res, int num_threads) const;
    // BFS levels from u in the partitioned convention (rank[u] = -1, level
    // >= 1, unreached INT_MAX); the serial reference returns a parent tree,
    // which is not unique -- the levels are.
    void solve_bfs(VID u, std::vector<VID>& rank) const;
    void solve_sssp(std::vector<int>& dist, VID src) const;
    void page_rank(std::vector<float>& pr_vals, float damping_factor, int num_iterations, int num_threads) const;
    void solve_kcore(std::vector<int>& core_numbers, int num_threads) const;
    void solve_mis(std::vector<int>& res, int num_threads) const;
    void solve_cdlp(std::vector<int>& labels, int max_iterations, int num_threads) const;

    pc_graph* device() const;  // uploads on first use

   private:
    friend class Partitioned_Graph;
    Partitioned_Graph& whole() const;
    size_t vertex_num = 0, edge_num = 0;
    std::vector<EID> csr_vlist;
    std::vector<VID> csr_elist;
    std::vector<Weight> csr_weight;
    mutable pc_graph* dev_ = nullptr;
    mutable Partitioned_Graph* whole_ = nullptr;
};

class Partitioned_Graph {
   public:
    // src/Graph.cpp:1017-1069; thread_num is accepted and ignored.
    Partitioned_Graph(const Graph& g, const std::vector<int>& vertex2partition, const int thread_num);
    ~Partitioned_Graph();
    Partitioned_Graph(const Partitioned_Graph&) = delete;
    Partitioned_Graph& operator=(const Partitioned_Graph&) = delete;

    size_t get_vertex_num() const { return n_; }
    size_t get_edge_num() const { return m_; }
    size_t get_partition_num() const;
    void reorder();
    void evaluate_partition() const;
    // The reference's layout (csr_vlist[k*n+u], partition-major csr_elist).
    void get_layout(std::vector<EID>& vlist, std::vector<VID>& elist) const;

    size_t solve_triangle_counting_galloping() const;
    size_t solve_triangle_counting_merge() const;
    // src/Graph.cpp:1222-1264 and 1291-1324
    size_t solve_friend_triangle_galloping(const VID root, const std::vector<VID>& nodes) const;
    size_t solve_friend_triangle_merge(const VID root, const std::vector<VID>& nodes) const;
    size_t solve_square_counting() const;
    void batch_cnt_common_neis_merge(const std::vector<std::pair<VID, VID>>& queries, std::vector<size_t>& res) const;
    void batch_cnt_common_neis_merge(const std::vector<std::vector<VID>>& queries, std::vector<size_t>& res) const;
    void batch_cnt_common_neis_galloping(const std::vector<std::pair<VID, VID>>& queries,
                                         std::vector<size_t>& res) const;
    void batch_cnt_common_neis_galloping(const std::vector<std::vector<VID>>& queries, std::vector<size_t>& res) const;
    void batch_cnt_common_neis_merge_fine_grained(const std::vector<std::pair<VID, VID>>& queries,
                                                  std::vector<size_t>& res) const;
    void batch_cnt_common_neis_galloping_fine_grained(const std::vector<std::pair<VID, VID>>& queries,
                                                      std::vector<size_t>& res) const;
    // The Graph:: formula c / (d_i + d_j - c); the reference's partitioned
    // version returns d_i + d_j - c without the division (src/Graph.cpp:2189-2194).
    void solve_jsim_merge(const std::vector<VID>& queries, std::vector<double>& res) const;
    void solve_jsim_galloping(const std::vector<VID>& queries, std::vector<double>& res) const;
    void solve_lcc_merge(std::vector<double>& res) const;
    void solve_lcc_galloping(std::vector<double>& res) const;
    void solve_bfs(VID u, std::vector<VID>& rank) const;
    void solve_sssp(VID src, std::vector<int>& dist) const;
    void page_rank(std::vector<float>& pr_vals, float damping_factor, int num_iterations) const;
    void solve_kcore(std::vector<int>& core_numbers) const;
    void solve_mis(std::vector<int>& res) const;
    void solve_cdlp(std::vector<int>& labels, int max_iterations) const;

    pc_pgraph* device() const { return pg_; }

   private:
    pc_pgraph* pg_ = nullptr;
    size_t n_ = 0, m_ = 0;
    bool weighted_ = false;
};

}  // namespace pc
