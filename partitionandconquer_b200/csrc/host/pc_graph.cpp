// Host classes with the reference's API (include/pc_graph.hpp).  Loading,
// preprocessing and partitioning are host C++; algorithms call the C ABI.
#include "../../../include/pc_graph.hpp"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <random>

#include "host_csr.hpp"

namespace pc {

static void check(pc_status s) {
    if (s != PC_OK) throw Error(s, pc_last_error());
}

// ---- Graph: construction ---------------------------------------------------------

// The text loader's parse (src/Graph.cpp:27-57): '#'/'%' comment lines,
// "u v" per line, self-loops skipped, ids shifted down by one unless a 0 id
// appears.  Returns the vertex count and the shifted endpoint streams.
static size_t parse_edge_text(const std::string& graphfile, std::vector<uint32_t>* s, std::vector<uint32_t>* d) {
    FILE* fp = fopen(graphfile.c_str(), "r");
    if (!fp) throw Error(PC_ERR_INVALID_INPUT, "cannot open " + graphfile);
    bool has_zero = false;
    size_t maxid = 0;
    std::vector<std::pair<VID, VID>> edges;
    char line[512];
    while (fgets(line, sizeof(line), fp) != nullptr) {
        if (line[0] == '#' || line[0] == '%') continue;
        long long u = 0, v = 0;
        const char* c = line;
        while (*c >= '0' && *c <= '9') u = u * 10 + (*c++ - '0');
        if (*c) ++c;
        while (*c >= '0' && *c <= '9') v = v * 10 + (*c++ - '0');
        if (u == 0 || v == 0) has_zero = true;
        if (u == v) continue;
        if ((size_t)u > maxid) maxid = (size_t)u;
        if ((size_t)v > maxid) maxid = (size_t)v;
        edges.emplace_back((VID)u, (VID)v);
    }
    fclose(fp);
    s->resize(edges.size());
    d->resize(edges.size());
    for (size_t i = 0; i < edges.size(); ++i) {
        (*s)[i] = (uint32_t)(edges[i].first - (has_zero ? 0 : 1));
        (*d)[i] = (uint32_t)(edges[i].second - (has_zero ? 0 : 1));
    }
    return maxid + (has_zero ? 1 : 0);
}

Graph::Graph(const std::string graphfile) {
    // src/Graph.cpp:27-90
    std::vector<uint32_t> s, d;
    vertex_num = parse_edge_text(graphfile, &s, &d);
    HostCSR g = build_symmetric_csr(vertex_num, s.size(), s.data(), d.data());
    csr_vlist.assign(g.vlist.begin(), g.vlist.end());
    csr_elist.assign(g.elist.begin(), g.elist.end());
    edge_num = csr_elist.size();
}

Graph::Graph(const std::string graphfile, OnDevice) {
    // the same parse; the adjacency build (src/Graph.cpp:59-85) runs on the GPU
    std::vector<uint32_t> s, d;
    vertex_num = parse_edge_text(graphfile, &s, &d);
    if (vertex_num == 0) return;
    pc_graph* h = nullptr;
    check(pc_graph_from_edges(s.data(), d.data(), s.size(), vertex_num, 0u, nullptr, &h));
    uint64_t n = 0, m = 0;
    int32_t w = 0;
    pc_graph_info(h, &n, &m, &w);
    csr_vlist.resize(n + 1);
    csr_elist.resize(m);
    const pc_status st = pc_graph_download(h, reinterpret_cast<uint64_t*>(csr_vlist.data()), csr_elist.data(), nullptr);
    if (st != PC_OK) {
        const std::string msg = pc_last_error();
        pc_graph_destroy(h);
        throw Error(st, msg);
    }
    edge_num = m;
    dev_ = h;  // the CSR is already on the device
}

Graph::Graph(const std::string csrdir, bool is_weighted) {
    HostCSR g;
    std::string err;
    if (!load_csr_binfiles(csrdir, is_weighted, &g, &err)) throw Error(PC_ERR_INVALID_INPUT, err);
    vertex_num = g.n;
    edge_num = g.m;
    csr_vlist.assign(g.vlist.begin(), g.vlist.end());
    csr_elist.assign(g.elist.begin(), g.elist.end());
    csr_weight.assign(g.weights.begin(), g.weights.end());
}

Graph::Graph(const std::vector<std::vector<VID>>& adj_list) {
    // src/Graph.cpp:139-149
    vertex_num = adj_list.size();
    csr_vlist.reserve(vertex_num + 1);
    csr_vlist.push_back(0);
    for (const auto& neis : adj_list) {
        csr_elist.insert(csr_elist.end(), neis.begin(), neis.end());
        csr_vlist.push_back(csr_elist.size());
    }
    edge_num = csr_elist.size();
}

Graph::Graph(std::vector<EID> vlist, std::vector<VID> elist, std::vector<Weight> weights)
    : csr_vlist(std::move(vlist)), csr_elist(std::move(elist)), csr_weight(std::move(weights)) {
    if (csr_vlist.empty()) throw Error(PC_ERR_INVALID_INPUT, "csr_vlist needs n+1 entries");
    vertex_num = csr_vlist.size() - 1;
    edge_num = csr_elist.size();
}

Graph::~Graph() {
    delete whole_;
    if (dev_) pc_graph_destroy(dev_);
}

pc_graph* Graph::device() const {
    if (!dev_) {
        check(pc_graph_create(reinterpret_cast<const uint64_t*>(csr_vlist.data()), csr_elist.data(),
                              csr_weight.empty() ? nullptr : csr_weight.data(), vertex_num, edge_num, 0, &dev_));
    }
    return dev_;
}

Partitioned_Graph& Graph::whole() const {
    if (!whole_) whole_ = new Partitioned_Graph(*this, std::vector<int>(), 1);
    return *whole_;
}

// ---- Graph: host accessors ---------------------------------------------------------

bool Graph::has_directed_edge(VID u, VID v) const {
    auto b = csr_elist.begin() + csr_vlist[u], e = csr_elist.begin() + csr_vlist[u + 1];
    auto it = std::lower_bound(b, e, v);
    return it != e && *it == v;
}

bool Graph::has_edge(VID u, VID v) const {
    return get_deg(u) < get_deg(v) ? has_directed_edge(u, v) : has_directed_edge(v, u);
}

size_t Graph::get_max_deg() const {
    size_t r = 0;
    for (size_t u = 0; u < vertex_num; ++u) r = std::max(r, get_deg((VID)u));
    return r;
}

void Graph::get_degs(std::vector<int>& degs) const {
    degs.resize(vertex_num);
    for (size_t u = 0; u < vertex_num; ++u) degs[u] = (int)get_deg((VID)u);
}

void Graph::get_neis(VID u, std::vector<VID>& neis) const {
    neis.assign(csr_elist.begin() + csr_vlist[u], csr_elist.begin() + csr_vlist[u + 1]);
}

void Graph::save_as_csr_binfile(const std::string vfile, const std::string efile) {
    std::ofstream a(vfile, std::ios::binary), b(efile, std::ios::binary);
    if (!a || !b) throw Error(PC_ERR_INVALID_INPUT, "cannot write " + vfile + " / " + efile);
    a.write(reinterpret_cast<const char*>(csr_vlist.data()), sizeof(EID) * csr_vlist.size());
    b.write(reinterpret_cast<const char*>(csr_elist.data()), sizeof(VID) * csr_elist.size());
}

void Graph::add_reference_weights() {
    // src/preprocess.cpp:10-37: for u < v draw rand() % floor(log2 n) + 1 from
    // the C library's generator (a fresh process starts it at seed 1); the
    // reverse entry copies the weight.  srand(1) reproduces a fresh process.
    const Weight max_weight = (Weight)std::log2((double)vertex_num);
    if (max_weight < 1) throw Error(PC_ERR_INVALID_INPUT, "graph too small for log2-range weights");
    csr_weight.assign(edge_num, 0);
    srand(1);
    for (size_t u = 0; u < vertex_num; ++u) {
        for (EID i = csr_vlist[u]; i < csr_vlist[u + 1]; ++i) {
            const VID v = csr_elist[i];
            if ((VID)u < v) {
                csr_weight[i] = rand() % max_weight + 1;
            } else {
                auto b = csr_elist.begin() + csr_vlist[v], e = csr_elist.begin() + csr_vlist[v + 1];
                csr_weight[i] = csr_weight[std::lower_bound(b, e, (VID)u) - csr_elist.begin()];
            }
        }
    }
}

void Graph::save_weight_binfile(const std::string wfile) const {
    std::ofstream a(wfile, std::ios::binary);
    if (!a) throw Error(PC_ERR_INVALID_INPUT, "cannot write " + wfile);
    a.write(reinterpret_cast<const char*>(csr_weight.data()), sizeof(Weight) * csr_weight.size());
}

void Graph::random_partition(const size_t part_num, std::vector<int>& v2p) {
    // src/Graph.cpp:564-570
    v2p.assign(vertex_num, 0);
    for (size_t u = 0; u < vertex_num; ++u) v2p[u] = rand() % (int)part_num;
}

void Graph::greedy_partition(const size_t P, std::vector<int>& v2p, uint64_t seed) {
    greedy_partition_host(vertex_num, reinterpret_cast<const uint64_t*>(csr_vlist.data()), csr_elist.data(), P, seed,
                          v2p);
}

// ---- Graph: algorithms (one partition) ------------------------------------------------

size_t Graph::solve_triangle_counting_galloping(const int) const { return whole().solve_triangle_counting_galloping(); }
size_t Graph::solve_triangle_counting_merge(const int) const { return whole().solve_triangle_counting_merge(); }
size_t Graph::solve_friend_triangle_galloping(const VID root, const std::vector<VID>& nodes, const int) const {
    return whole().solve_friend_triangle_galloping(root, nodes);
}
size_t Graph::solve_friend_triangle_merge(const VID root, const std::vector<VID>& nodes, const int) const {
    return whole().solve_friend_triangle_merge(root, nodes);
}
void Graph::batch_cnt_common_neis_merge(const std::vector<std::pair<VID, VID>>& q, std::vector<size_t>& r, int) const {
    whole().batch_cnt_common_neis_merge(q, r);
}
void Graph::batch_cnt_common_neis_merge(const std::vector<std::vector<VID>>& q, std::vector<size_t>& r, int) const {
    whole().batch_cnt_common_neis_merge(q, r);
}
void Graph::batch_cnt_common_neis_galloping(const std::vector<std::pair<VID, VID>>& q, std::vector<size_t>& r,
                                            int) const {
    whole().batch_cnt_common_neis_merge(q, r);
}
void Graph::solve_jsim_merge(const std::vector<VID>& q, std::vector<double>& r, int) const { whole().solve_jsim_merge(q, r); }
void Graph::solve_jsim_galloping(const std::vector<VID>& q, std::vector<double>& r, int) const {
    whole().solve_jsim_merge(q, r);
}
void Graph::solve_lcc_merge(std::vector<double>& r, int) const { whole().solve_lcc_merge(r); }
void Graph::solve_lcc_galloping(std::vector<double>& r, int) const { whole().solve_lcc_galloping(r); }
void Graph::solve_bfs(VID u, std::vector<VID>& rank) const { whole().solve_bfs(u, rank); }
void Graph::solve_sssp(std::vector<int>& dist, VID src) const { whole().solve_sssp(src, dist); }
void Graph::page_rank(std::vector<float>& pr, float damping, int iters, int) const {
    // src/Graph.cpp:534-554: starts from the caller's vector
    if (pr.size() != vertex_num) throw Error(PC_ERR_INVALID_INPUT, "pr_vals must have n entries");
    std::vector<float> out(vertex_num);
    check(pc_pagerank(whole().device(), damping, iters, pr.data(), out.data()));
    pr.swap(out);
}
void Graph::solve_kcore(std::vector<int>& core, int) const { whole().solve_kcore(core); }
void Graph::solve_mis(std::vector<int>& res, int) const { whole().solve_mis(res); }
void Graph::solve_cdlp(std::vector<int>& labels, int iters, int) const { whole().solve_cdlp(labels, iters); }

// ---- Partitioned_Graph -------------------------------------------------------------------

Partitioned_Graph::Partitioned_Graph(const Graph& g, const std::vector<int>& v2p, const int) {
    if (!v2p.empty() && v2p.size() != g.vertex_num)
        throw Error(PC_ERR_INVALID_INPUT, "vertex2partition needs one entry per vertex");
    n_ = g.vertex_num;
    m_ = g.edge_num;
    weighted_ = g.is_weighted();
    check(pc_partition(g.device(), v2p.empty() ? nullptr : v2p.data(), &pg_));
}

Partitioned_Graph::~Partitioned_Graph() {
    if (pg_) pc_pgraph_destroy(pg_);
}

size_t Partitioned_Graph::get_partition_num() const {
    int32_t p = 0;
    check(pc_pgraph_info(pg_, nullptr, nullptr, &p));
    return (size_t)p;
}

void Partitioned_Graph::reorder() { check(pc_pgraph_reorder(pg_)); }

void Partitioned_Graph::evaluate_partition() const {
    int64_t mpd = 0, md = 0;
    double r = 0;
    check(pc_pgraph_evaluate(pg_, &mpd, &md, &r));
    printf("max part deg: %lld, max deg: %lld, balance ratio: %f\n", (long long)mpd, (long long)md, r);
}

void Partitioned_Graph::get_layout(std::vector<EID>& vlist, std::vector<VID>& elist) const {
    vlist.resize(get_partition_num() * n_ + 1);
    elist.resize(m_);
    check(pc_pgraph_layout(pg_, reinterpret_cast<uint64_t*>(vlist.data()), elist.data(), nullptr));
}

size_t Partitioned_Graph::solve_triangle_counting_galloping() const {
    uint64_t c = 0;
    check(pc_tc(pg_, PC_METHOD_GALLOPING, &c));
    return (size_t)c;
}

size_t Partitioned_Graph::solve_triangle_counting_merge() const {
    uint64_t c = 0;
    check(pc_tc(pg_, PC_METHOD_MERGE, &c));
    return (size_t)c;
}

size_t Partitioned_Graph::solve_friend_triangle_merge(const VID root, const std::vector<VID>& nodes) const {
    uint64_t c = 0;
    check(pc_friend_triangle(pg_, root, nodes.data(), nodes.size(), &c));
    return c;
}

size_t Partitioned_Graph::solve_friend_triangle_galloping(const VID root, const std::vector<VID>& nodes) const {
    return solve_friend_triangle_merge(root, nodes);
}

size_t Partitioned_Graph::solve_square_counting() const {
    uint64_t c = 0;
    check(pc_square_count(pg_, &c));
    return c;
}

void Partitioned_Graph::batch_cnt_common_neis_merge(const std::vector<std::pair<VID, VID>>& q,
                                                    std::vector<size_t>& res) const {
    std::vector<int32_t> flat(2 * q.size());
    for (size_t i = 0; i < q.size(); ++i) { flat[2 * i] = q[i].first; flat[2 * i + 1] = q[i].second; }
    std::vector<uint64_t> out(q.size());
    check(pc_batch_count_pairs(pg_, flat.data(), q.size(), out.data()));
    res.assign(out.begin(), out.end());
}

void Partitioned_Graph::batch_cnt_common_neis_merge(const std::vector<std::vector<VID>>& q,
                                                    std::vector<size_t>& res) const {
    std::vector<int32_t> ids;
    std::vector<uint64_t> offs(1, 0);
    for (const auto& s : q) {
        ids.insert(ids.end(), s.begin(), s.end());
        offs.push_back(ids.size());
    }
    std::vector<uint64_t> out(q.size());
    check(pc_batch_count_sets(pg_, ids.data(), offs.data(), q.size(), out.data()));
    res.assign(out.begin(), out.end());
}

void Partitioned_Graph::batch_cnt_common_neis_galloping(const std::vector<std::pair<VID, VID>>& q,
                                                        std::vector<size_t>& r) const {
    batch_cnt_common_neis_merge(q, r);
}
void Partitioned_Graph::batch_cnt_common_neis_galloping(const std::vector<std::vector<VID>>& q,
                                                        std::vector<size_t>& r) const {
    batch_cnt_common_neis_merge(q, r);
}
void Partitioned_Graph::batch_cnt_common_neis_merge_fine_grained(const std::vector<std::pair<VID, VID>>& q,
                                                                 std::vector<size_t>& r) const {
    batch_cnt_common_neis_merge(q, r);
}
void Partitioned_Graph::batch_cnt_common_neis_galloping_fine_grained(const std::vector<std::pair<VID, VID>>& q,
                                                                     std::vector<size_t>& r) const {
    batch_cnt_common_neis_merge(q, r);
}

void Partitioned_Graph::solve_jsim_merge(const std::vector<VID>& q, std::vector<double>& res) const {
    res.assign(q.size() * q.size(), 0.0);
    check(pc_jaccard_queries(pg_, q.data(), (int32_t)q.size(), res.data()));
}
void Partitioned_Graph::solve_jsim_galloping(const std::vector<VID>& q, std::vector<double>& r) const {
    solve_jsim_merge(q, r);
}

void Partitioned_Graph::solve_lcc_merge(std::vector<double>& res) const {
    res.assign(n_, 0.0);
    check(pc_lcc(pg_, PC_METHOD_MERGE, res.data()));
}
void Partitioned_Graph::solve_lcc_galloping(std::vector<double>& res) const {
    res.assign(n_, 0.0);
    check(pc_lcc(pg_, PC_METHOD_GALLOPING, res.data()));
}

void Partitioned_Graph::solve_bfs(VID u, std::vector<VID>& rank) const {
    rank.assign(n_, INT_MAX);
    check(pc_bfs(pg_, u, rank.data()));
}

void Partitioned_Graph::solve_sssp(VID src, std::vector<int>& dist) const {
    // the reference fills dist with INT_MAX / 2 itself or expects it pre-filled
    // (src/test.cpp:202-203); the result is the same either way.
    dist.assign(n_, INT_MAX / 2);
    check(pc_sssp(pg_, src, dist.data()));
}

void Partitioned_Graph::page_rank(std::vector<float>& pr, float damping, int iters) const {
    // src/Graph.cpp:1555-1602 ignores the caller's initial values
    pr.assign(n_, 0.f);
    check(pc_pagerank(pg_, damping, iters, nullptr, pr.data()));
}

void Partitioned_Graph::solve_kcore(std::vector<int>& core) const {
    core.assign(n_, 0);
    int32_t largest = 0;
    check(pc_kcore(pg_, core.data(), &largest));
}

void Partitioned_Graph::solve_mis(std::vector<int>& res) const {
    res.assign(n_, 0);
    check(pc_mis(pg_, res.data()));
}

void Partitioned_Graph::solve_cdlp(std::vector<int>& labels, int iters) const {
    if (labels.size() != n_) throw Error(PC_ERR_INVALID_INPUT, "labels must have n entries");
    check(pc_cdlp(pg_, iters, labels.data()));
}

}  // namespace pc
