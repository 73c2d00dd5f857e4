// Host-side CSR graph container and builders (C++17 + OpenMP).
//
// The CSR follows the reference's binary format (Graph::Graph(csrdir, bool),
// src/Graph.cpp:92-137): offsets are uint64 (EID, n+1 entries), neighbour ids
// are int32 (VID, m entries, each list sorted ascending, no duplicates, no
// self-loops), weights are int32 (m entries, symmetric).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace pc {

struct HostCSR {
    uint64_t n = 0;
    uint64_t m = 0;
    std::vector<uint64_t> vlist;   // n + 1
    std::vector<int32_t> elist;    // m
    std::vector<int32_t> weights;  // m or empty
};

// Symmetrise an edge list: every (u, v) with u != v yields u->v and v->u;
// rows are sorted and de-duplicated.  n is fixed by the caller (isolated
// vertices are kept).  Semantics follow the text loader's adjacency build
// (src/Graph.cpp:59-85) without its id shift.
HostCSR build_symmetric_csr(uint64_t n, uint64_t nedges, const uint32_t* src, const uint32_t* dst);

// Relabel vertices by descending degree, ties by ascending id, and rebuild
// the sorted CSR.  Returns old->new in perm_out when non-null.
HostCSR relabel_by_degree(const HostCSR& g, std::vector<int32_t>* old2new = nullptr);

// Relabel with an explicit old->new permutation (rows re-sorted).
HostCSR relabel(const HostCSR& g, const std::vector<int32_t>& old2new);

// Synthetic generators (seeded, deterministic, identical to the device ones).
HostCSR gen_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, bool degree_relabel);
HostCSR gen_er(uint32_t scale, uint64_t nedges, uint64_t seed, bool degree_relabel);
HostCSR gen_chung_lu(uint32_t scale, uint64_t nedges, double beta, uint64_t dmax, uint64_t seed, bool degree_relabel);

// G RMAT graphs packed in one arena (graph g: RMAT seed g; scale and edge
// factor drawn from `seed`), each degree-relabelled; voff gets G+1 offsets.
HostCSR gen_rmat_batch(uint32_t G, uint32_t smin, uint32_t smax, uint32_t emin, uint32_t emax, uint64_t seed,
                       std::vector<uint64_t>* voff);

// Raw edge streams (before symmetrisation), for the device-side builder tests.
void rmat_edges(uint32_t scale, uint64_t nedges, uint64_t seed, uint32_t* src, uint32_t* dst);

// Symmetric integer weights in [1, wmax] keyed on the unordered endpoint pair.
void add_weights(HostCSR& g, uint64_t seed, int32_t wmax);

// Validation of the boundary input: monotone offsets, ids in range, sorted
// rows, weights length.  Returns an empty string when valid.
std::string validate_csr(uint64_t n, uint64_t m, const uint64_t* vlist, const int32_t* elist, bool require_sorted);

// Graph::greedy_partition (src/Graph.cpp:898-967) with a seeded engine in
// place of random_device and rand().
void greedy_partition_host(uint64_t n, const uint64_t* vlist, const int32_t* elist, size_t P, uint64_t seed,
                           std::vector<int>& v2p);

// Binary files in the reference format.
bool save_csr_binfiles(const HostCSR& g, const std::string& dir, std::string* err);
bool load_csr_binfiles(const std::string& dir, bool weighted, HostCSR* g, std::string* err);

}  // namespace pc
