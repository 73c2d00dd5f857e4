// Host CSR builders, seeded generators and reference-format binary files.
#include "host_csr.hpp"

#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <numeric>
#include <random>

#include "../synth_rng.h"

namespace pc {

namespace {

// Exclusive prefix sum of counts[0..n) into off[0..n] (off[n] = total), parallel.
void exclusive_scan_u64(const std::vector<uint64_t>& counts, std::vector<uint64_t>& off) {
    const uint64_t n = counts.size();
    off.assign(n + 1, 0);
    const int nt = omp_get_max_threads();
    std::vector<uint64_t> part(nt + 1, 0);
    int used = 1;
#pragma omp parallel num_threads(nt)
    {
        // the team can be smaller than nt (nested inside another parallel region)
        const int T = omp_get_num_threads(), t = omp_get_thread_num();
        uint64_t lo = n * t / T, hi = n * (t + 1) / T, s = 0;
        for (uint64_t i = lo; i < hi; ++i) s += counts[i];
        part[t + 1] = s;
#pragma omp barrier
#pragma omp single
        {
            used = T;
            for (int i = 0; i < T; ++i) part[i + 1] += part[i];
        }
        s = part[t];
        for (uint64_t i = lo; i < hi; ++i) {
            off[i] = s;
            s += counts[i];
        }
    }
    off[n] = part[used];
}

}  // namespace

HostCSR build_symmetric_csr(uint64_t n, uint64_t nedges, const uint32_t* src, const uint32_t* dst) {
    HostCSR g;
    g.n = n;
    std::vector<std::atomic<uint32_t>> deg(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) deg[i].store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < (int64_t)nedges; ++k) {
        uint32_t u = src[k], v = dst[k];
        if (u == v) continue;
        deg[u].fetch_add(1, std::memory_order_relaxed);
        deg[v].fetch_add(1, std::memory_order_relaxed);
    }
    std::vector<uint64_t> cnt(n), off;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) cnt[i] = deg[i].load(std::memory_order_relaxed);
    exclusive_scan_u64(cnt, off);
    std::vector<int32_t> col(off[n]);
    // cursors reuse the atomic degree array
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) deg[i].store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < (int64_t)nedges; ++k) {
        uint32_t u = src[k], v = dst[k];
        if (u == v) continue;
        col[off[u] + deg[u].fetch_add(1, std::memory_order_relaxed)] = (int32_t)v;
        col[off[v] + deg[v].fetch_add(1, std::memory_order_relaxed)] = (int32_t)u;
    }
    std::vector<uint64_t> ucnt(n);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        int32_t* b = col.data() + off[i];
        int32_t* e = col.data() + off[i + 1];
        std::sort(b, e);
        ucnt[i] = (uint64_t)(std::unique(b, e) - b);
    }
    exclusive_scan_u64(ucnt, g.vlist);
    g.m = g.vlist[n];
    g.elist.resize(g.m);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t i = 0; i < (int64_t)n; ++i)
        std::memcpy(g.elist.data() + g.vlist[i], col.data() + off[i], ucnt[i] * sizeof(int32_t));
    return g;
}

HostCSR relabel(const HostCSR& g, const std::vector<int32_t>& old2new) {
    const uint64_t n = g.n;
    HostCSR r;
    r.n = n;
    r.m = g.m;
    std::vector<int32_t> new2old(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) new2old[old2new[i]] = (int32_t)i;
    std::vector<uint64_t> cnt(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        int32_t o = new2old[i];
        cnt[i] = g.vlist[o + 1] - g.vlist[o];
    }
    exclusive_scan_u64(cnt, r.vlist);
    r.elist.resize(g.m);
    const bool w = !g.weights.empty();
    if (w) r.weights.resize(g.m);
#pragma omp parallel
    {
        std::vector<std::pair<int32_t, int32_t>> tmp;
#pragma omp for schedule(dynamic, 1024)
        for (int64_t i = 0; i < (int64_t)n; ++i) {
            int32_t o = new2old[i];
            uint64_t b = g.vlist[o], e = g.vlist[o + 1], d = r.vlist[i];
            if (!w) {
                for (uint64_t k = b; k < e; ++k) r.elist[d + (k - b)] = old2new[g.elist[k]];
                std::sort(r.elist.begin() + d, r.elist.begin() + d + (e - b));
            } else {
                tmp.clear();
                for (uint64_t k = b; k < e; ++k) tmp.emplace_back(old2new[g.elist[k]], g.weights[k]);
                std::sort(tmp.begin(), tmp.end());
                for (uint64_t k = 0; k < tmp.size(); ++k) {
                    r.elist[d + k] = tmp[k].first;
                    r.weights[d + k] = tmp[k].second;
                }
            }
        }
    }
    return r;
}

HostCSR relabel_by_degree(const HostCSR& g, std::vector<int32_t>* old2new_out) {
    const uint64_t n = g.n;
    // key = (max_deg - deg) << 32 | id: ascending key = descending degree, ties by id.
    std::vector<uint64_t> key(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        uint64_t d = g.vlist[i + 1] - g.vlist[i];
        key[i] = ((0xFFFFFFFFull - d) << 32) | (uint64_t)i;
    }
    // parallel sort: sort per-thread blocks then merge pairwise
    int nt = omp_get_max_threads();
    std::vector<uint64_t> bounds(nt + 1);
    for (int t = 0; t <= nt; ++t) bounds[t] = n * t / nt;
#pragma omp parallel for num_threads(nt)
    for (int t = 0; t < nt; ++t) std::sort(key.begin() + bounds[t], key.begin() + bounds[t + 1]);
    for (int width = 1; width < nt; width *= 2) {
#pragma omp parallel for num_threads(nt)
        for (int t = 0; t < nt; t += 2 * width) {
            if (t + width < nt) {
                uint64_t lo = bounds[t], mid = bounds[t + width], hi = bounds[std::min(t + 2 * width, nt)];
                std::inplace_merge(key.begin() + lo, key.begin() + mid, key.begin() + hi);
            }
        }
    }
    std::vector<int32_t> old2new(n);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < (int64_t)n; ++r) old2new[(uint32_t)(key[r] & 0xFFFFFFFFull)] = (int32_t)r;
    HostCSR out = relabel(g, old2new);
    if (old2new_out) old2new_out->swap(old2new);
    return out;
}

void rmat_edges(uint32_t scale, uint64_t nedges, uint64_t seed, uint32_t* src, uint32_t* dst) {
    const uint64_t key = pc_graph_key(seed, PC_GEN_RMAT);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < (int64_t)nedges; ++k) pc_rmat_edge(key, (uint64_t)k, scale, &src[k], &dst[k]);
}

HostCSR gen_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, bool degree_relabel) {
    const uint64_t n = 1ull << scale, ne = n * edge_factor;
    std::vector<uint32_t> s(ne), d(ne);
    rmat_edges(scale, ne, seed, s.data(), d.data());
    HostCSR g = build_symmetric_csr(n, ne, s.data(), d.data());
    std::vector<uint32_t>().swap(s);
    std::vector<uint32_t>().swap(d);
    return degree_relabel ? relabel_by_degree(g) : g;
}

HostCSR gen_rmat_batch(uint32_t G, uint32_t smin, uint32_t smax, uint32_t emin, uint32_t emax, uint64_t seed,
                       std::vector<uint64_t>* voff) {
    const uint64_t key = pc_graph_key(seed, PC_GEN_BATCH);
    std::vector<HostCSR> gs(G);
    // one graph per thread (the builders' own parallel regions run nested, serially)
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t g = 0; g < (int64_t)G; ++g) {
        const uint32_t scale = smin + (uint32_t)(pc_draw(key, 2 * (uint64_t)g) % (uint64_t)(smax - smin + 1));
        const uint32_t ef = emin + (uint32_t)(pc_draw(key, 2 * (uint64_t)g + 1) % (uint64_t)(emax - emin + 1));
        gs[g] = gen_rmat(scale, ef, (uint64_t)g, true);
    }
    voff->assign(G + 1, 0);
    std::vector<uint64_t> eoff(G + 1, 0);
    for (uint32_t g = 0; g < G; ++g) {
        (*voff)[g + 1] = (*voff)[g] + gs[g].n;
        eoff[g + 1] = eoff[g] + gs[g].m;
    }
    HostCSR a;
    a.n = (*voff)[G];
    a.m = eoff[G];
    a.vlist.resize(a.n + 1);
    a.elist.resize(a.m);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t g = 0; g < (int64_t)G; ++g) {
        const HostCSR& x = gs[g];
        const uint64_t vb = (*voff)[g], eb = eoff[g];
        for (uint64_t u = 0; u < x.n; ++u) a.vlist[vb + u] = eb + x.vlist[u];
        for (uint64_t k = 0; k < x.m; ++k) a.elist[eb + k] = x.elist[k] + (int32_t)vb;
    }
    a.vlist[a.n] = a.m;
    return a;
}

HostCSR gen_er(uint32_t scale, uint64_t nedges, uint64_t seed, bool degree_relabel) {
    const uint64_t n = 1ull << scale;
    const uint64_t key = pc_graph_key(seed, PC_GEN_ER);
    std::vector<uint32_t> s(nedges), d(nedges);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < (int64_t)nedges; ++k) pc_er_edge(key, (uint64_t)k, scale, &s[k], &d[k]);
    HostCSR g = build_symmetric_csr(n, nedges, s.data(), d.data());
    return degree_relabel ? relabel_by_degree(g) : g;
}

HostCSR gen_chung_lu(uint32_t scale, uint64_t nedges, double beta, uint64_t dmax, uint64_t seed, bool degree_relabel) {
    // Expected-degree (Chung-Lu) model: w_i = (i + i0)^(-1/(beta-1)); i0 is set
    // by bisection so that the expected degree of vertex 0, 2*nedges*w_0/sum(w),
    // equals dmax.  Endpoints are drawn by inverse CDF over a 2^62 fixed-point table.
    const uint64_t n = 1ull << scale;
    const double alpha = 1.0 / (beta - 1.0);
    auto expected_max = [&](double i0) {
        double s = 0.0;
        for (uint64_t i = 0; i < n; ++i) s += std::pow((double)i + i0, -alpha);
        return 2.0 * (double)nedges * std::pow(i0, -alpha) / s;
    };
    double lo = 1e-3, hi = (double)n;
    for (int it = 0; it < 60; ++it) {
        double mid = std::sqrt(lo * hi);
        if (expected_max(mid) > (double)dmax) lo = mid; else hi = mid;
    }
    const double i0 = hi;
    std::vector<double> w(n);
    double tot = 0.0;
    for (uint64_t i = 0; i < n; ++i) { w[i] = std::pow((double)i + i0, -alpha); tot += w[i]; }
    std::vector<uint64_t> cdf(n);
    double acc = 0.0;
    const double scale62 = 4611686018427387904.0;  // 2^62
    for (uint64_t i = 0; i < n; ++i) {
        acc += w[i];
        cdf[i] = (uint64_t)std::min(scale62, std::floor(acc / tot * scale62));
    }
    cdf[n - 1] = (uint64_t)scale62;
    const uint64_t key = pc_graph_key(seed, PC_GEN_CHUNG_LU);
    std::vector<uint32_t> s(nedges), d(nedges);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < (int64_t)nedges; ++k) {
        for (int e = 0; e < 2; ++e) {
            uint64_t r = pc_draw(key, ((uint64_t)k << 1) | (uint64_t)e) >> 2;  // [0, 2^62)
            uint32_t idx = (uint32_t)(std::upper_bound(cdf.begin(), cdf.end(), r) - cdf.begin());
            if (idx >= n) idx = (uint32_t)(n - 1);
            (e ? d : s)[k] = idx;
        }
    }
    HostCSR g = build_symmetric_csr(n, nedges, s.data(), d.data());
    return degree_relabel ? relabel_by_degree(g) : g;
}

void add_weights(HostCSR& g, uint64_t seed, int32_t wmax) {
    const uint64_t key = pc_graph_key(seed, PC_GEN_WEIGHT);
    g.weights.resize(g.m);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t u = 0; u < (int64_t)g.n; ++u)
        for (uint64_t k = g.vlist[u]; k < g.vlist[u + 1]; ++k)
            g.weights[k] = pc_edge_weight(key, (uint32_t)u, (uint32_t)g.elist[k], wmax);
}

std::string validate_csr(uint64_t n, uint64_t m, const uint64_t* vlist, const int32_t* elist, bool require_sorted) {
    if (n >= (1ull << 31)) return "vertex count does not fit the int32 vertex id type";
    if (!vlist) return "null offset array";
    if (m > 0 && !elist) return "null neighbour array";
    if (vlist[0] != 0) return "csr_vlist[0] must be 0";
    if (vlist[n] != m) return "csr_vlist[n] must equal the edge count";
    std::atomic<int> bad(0);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t u = 0; u < (int64_t)n; ++u) {
        if (bad.load(std::memory_order_relaxed)) continue;
        uint64_t b = vlist[u], e = vlist[u + 1];
        if (e < b || e > m) { bad.store(1); continue; }
        for (uint64_t k = b; k < e; ++k) {
            int32_t v = elist[k];
            if (v < 0 || (uint64_t)v >= n) { bad.store(2); break; }
            if (require_sorted && k > b && elist[k - 1] >= v) { bad.store(3); break; }
        }
    }
    switch (bad.load()) {
        case 1: return "csr_vlist is not monotone";
        case 2: return "neighbour id out of range";
        case 3: return "neighbour lists must be strictly ascending";
        default: return "";
    }
}

namespace {
bool write_file(const std::string& path, const void* p, size_t bytes, std::string* err) {
    std::ofstream f(path, std::ios::binary);
    if (!f) { if (err) *err = "cannot open " + path + " for writing"; return false; }
    f.write(reinterpret_cast<const char*>(p), (std::streamsize)bytes);
    if (!f) { if (err) *err = "short write to " + path; return false; }
    return true;
}
template <class T>
bool read_file(const std::string& path, std::vector<T>* v, std::string* err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) { if (err) *err = "cannot open " + path; return false; }
    f.seekg(0, std::ios::end);
    std::streamsize size = f.tellg();
    f.seekg(0, std::ios::beg);
    if (size % (std::streamsize)sizeof(T) != 0) { if (err) *err = path + ": size is not a multiple of the element size"; return false; }
    v->resize((size_t)size / sizeof(T));
    f.read(reinterpret_cast<char*>(v->data()), size);
    if (!f) { if (err) *err = "short read from " + path; return false; }
    return true;
}
}  // namespace

bool save_csr_binfiles(const HostCSR& g, const std::string& dir, std::string* err) {
    if (!write_file(dir + "/csr_vlist.bin", g.vlist.data(), g.vlist.size() * 8, err)) return false;
    if (!write_file(dir + "/csr_elist.bin", g.elist.data(), g.elist.size() * 4, err)) return false;
    if (!g.weights.empty() && !write_file(dir + "/csr_weight.bin", g.weights.data(), g.weights.size() * 4, err)) return false;
    return true;
}

bool load_csr_binfiles(const std::string& dir, bool weighted, HostCSR* g, std::string* err) {
    if (!read_file(dir + "/csr_vlist.bin", &g->vlist, err)) return false;
    if (g->vlist.empty()) { if (err) *err = "empty csr_vlist.bin"; return false; }
    if (!read_file(dir + "/csr_elist.bin", &g->elist, err)) return false;
    g->n = g->vlist.size() - 1;
    g->m = g->elist.size();
    if (weighted) {
        if (!read_file(dir + "/csr_weight.bin", &g->weights, err)) return false;
        if (g->weights.size() != g->m) { if (err) *err = "csr_weight.bin length differs from csr_elist.bin"; return false; }
    }
    std::string e = validate_csr(g->n, g->m, g->vlist.data(), g->elist.data(), false);
    if (!e.empty()) { if (err) *err = e; return false; }
    return true;
}


void greedy_partition_host(uint64_t n, const uint64_t* vlist, const int32_t* elist, size_t P, uint64_t seed,
                           std::vector<int>& v2p) {
    // src/Graph.cpp:898-967 with one seeded engine in place of random_device
    // and rand(), so the result is reproducible.
    std::vector<std::pair<int32_t, int>> deg(n);
    v2p.assign(n, -1);
    for (uint64_t i = 0; i < n; ++i) deg[i] = {(int32_t)i, (int)(vlist[i + 1] - vlist[i])};
    std::sort(deg.begin(), deg.end(),
              [](std::pair<int32_t, int> a, std::pair<int32_t, int> b) { return a.second > b.second; });
    std::mt19937 rng((uint32_t)seed);
    std::vector<int> cnt(P);
    std::vector<int32_t> free_nbrs;
    std::vector<int> plist(P);
    for (const auto& item : deg) {
        std::fill(cnt.begin(), cnt.end(), 0);
        free_nbrs.clear();
        const int32_t u = item.first;
        for (uint64_t i = vlist[u]; i < vlist[u + 1]; ++i) {
            const int32_t v = elist[i];
            if (v2p[v] > -1) cnt[v2p[v]]++;
            else free_nbrs.push_back(v);
        }
        if (free_nbrs.empty()) continue;
        std::shuffle(free_nbrs.begin(), free_nbrs.end(), rng);
        const int ulb = item.second / (int)P;
        for (size_t k = 0; k < P; ++k) plist[k] = std::max(0, ulb - cnt[k]);
        const long long psum = std::accumulate(plist.begin(), plist.end(), 0LL);
        size_t ptr = 0;
        if (psum > 0) {
            for (size_t k = 0; k < P; ++k) {
                const size_t len = (size_t)((long long)plist[k] * (long long)free_nbrs.size() / psum);
                for (size_t j = 0; j < len && ptr < free_nbrs.size(); ++j) v2p[free_nbrs[ptr++]] = (int)k;
            }
        }
        for (; ptr < free_nbrs.size(); ++ptr) v2p[free_nbrs[ptr]] = (int)(rng() % P);
    }
    for (uint64_t u = 0; u < n; ++u)
        if (v2p[u] == -1) v2p[u] = (int)(rng() % P);
}

}  // namespace pc
