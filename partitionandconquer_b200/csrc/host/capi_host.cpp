// C ABI of the host-side helpers: seeded synthetic graphs and the reference's
// binary CSR files.  Errors are reported through pc_last_error() like the
// device entry points.
#include <algorithm>
#include <cstring>
#include <new>
#include <string>

#include "../../../include/pc.h"
#include "../synth_rng.h"
#include "host_csr.hpp"

namespace pc {
void set_error(const std::string& msg);
void clear_error();
pc_status fail(pc_status st, const std::string& msg);
}  // namespace pc

struct pc_host_csr {
    pc::HostCSR g;
};

using pc::fail;

extern "C" {

static pc_status wrap(pc::HostCSR&& g, pc_host_csr** out) {
    pc_host_csr* h = new (std::nothrow) pc_host_csr();
    if (!h) return fail(PC_ERR_OOM, "host allocation failed");
    h->g = std::move(g);
    *out = h;
    return PC_OK;
}

pc_status pc_synth_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, int32_t relabel, pc_host_csr** out) {
    pc::clear_error();
    if (!out) return fail(PC_ERR_INVALID_INPUT, "out is null");
    if (scale < 1 || scale > 30 || edge_factor < 1) return fail(PC_ERR_INVALID_INPUT, "scale must be in [1,30], edge_factor >= 1");
    try {
        return wrap(pc::gen_rmat(scale, edge_factor, seed, relabel != 0), out);
    } catch (const std::bad_alloc&) {
        return fail(PC_ERR_OOM, "host allocation failed");
    }
}

pc_status pc_synth_er(uint32_t scale, uint64_t nedges, uint64_t seed, int32_t relabel, pc_host_csr** out) {
    pc::clear_error();
    if (!out) return fail(PC_ERR_INVALID_INPUT, "out is null");
    if (scale < 1 || scale > 30) return fail(PC_ERR_INVALID_INPUT, "scale must be in [1,30]");
    try {
        return wrap(pc::gen_er(scale, nedges, seed, relabel != 0), out);
    } catch (const std::bad_alloc&) {
        return fail(PC_ERR_OOM, "host allocation failed");
    }
}

pc_status pc_synth_chung_lu(uint32_t scale, uint64_t nedges, double beta, uint64_t dmax, uint64_t seed, int32_t relabel,
                            pc_host_csr** out) {
    pc::clear_error();
    if (!out) return fail(PC_ERR_INVALID_INPUT, "out is null");
    if (scale < 1 || scale > 30 || !(beta > 1.0) || dmax < 1) return fail(PC_ERR_INVALID_INPUT, "bad Chung-Lu parameters");
    try {
        return wrap(pc::gen_chung_lu(scale, nedges, beta, dmax, seed, relabel != 0), out);
    } catch (const std::bad_alloc&) {
        return fail(PC_ERR_OOM, "host allocation failed");
    }
}

pc_status pc_synth_add_weights(pc_host_csr* g, uint64_t seed, int32_t wmax) {
    pc::clear_error();
    if (!g || wmax < 1) return fail(PC_ERR_INVALID_INPUT, "bad argument");
    pc::add_weights(g->g, seed, wmax);
    return PC_OK;
}

pc_status pc_host_csr_arrays(const pc_host_csr* g, uint64_t* n, uint64_t* m, const uint64_t** vlist,
                             const int32_t** elist, const int32_t** weights) {
    pc::clear_error();
    if (!g) return fail(PC_ERR_INVALID_INPUT, "null host csr");
    if (n) *n = g->g.n;
    if (m) *m = g->g.m;
    if (vlist) *vlist = g->g.vlist.data();
    if (elist) *elist = g->g.elist.data();
    if (weights) *weights = g->g.weights.empty() ? nullptr : g->g.weights.data();
    return PC_OK;
}

pc_status pc_host_csr_load(const char* dir, int32_t weighted, pc_host_csr** out) {
    pc::clear_error();
    if (!dir || !out) return fail(PC_ERR_INVALID_INPUT, "null argument");
    pc::HostCSR g;
    std::string err;
    if (!pc::load_csr_binfiles(dir, weighted != 0, &g, &err)) return fail(PC_ERR_INVALID_INPUT, err);
    return wrap(std::move(g), out);
}

pc_status pc_host_csr_save(const pc_host_csr* g, const char* dir) {
    pc::clear_error();
    if (!g || !dir) return fail(PC_ERR_INVALID_INPUT, "null argument");
    std::string err;
    if (!pc::save_csr_binfiles(g->g, dir, &err)) return fail(PC_ERR_INVALID_INPUT, err);
    return PC_OK;
}

pc_status pc_host_csr_from_arrays(const uint64_t* vlist, const int32_t* elist, const int32_t* weights, uint64_t n,
                                  uint64_t m, pc_host_csr** out) {
    pc::clear_error();
    if (!vlist || (m && !elist) || !out) return fail(PC_ERR_INVALID_INPUT, "null argument");
    pc::HostCSR g;
    g.n = n;
    g.m = m;
    g.vlist.assign(vlist, vlist + n + 1);
    g.elist.assign(elist, elist + m);
    if (weights) g.weights.assign(weights, weights + m);
    std::string e = pc::validate_csr(n, m, g.vlist.data(), g.elist.data(), false);
    if (!e.empty()) return fail(PC_ERR_INVALID_INPUT, e);
    return wrap(std::move(g), out);
}

pc_status pc_host_csr_free(pc_host_csr* g) {
    pc::clear_error();
    delete g;
    return PC_OK;
}

pc_status pc_synth_rmat_batch(uint32_t G, uint32_t smin, uint32_t smax, uint32_t emin, uint32_t emax, uint64_t seed,
                              pc_host_csr** out, uint64_t* voff) {
    pc::clear_error();
    if (!out || !voff || G == 0) return fail(PC_ERR_INVALID_INPUT, "bad argument");
    if (smin < 1 || smax > 26 || smin > smax || emin < 1 || emin > emax)
        return fail(PC_ERR_INVALID_INPUT, "bad scale or edge-factor range");
    try {
        std::vector<uint64_t> v;
        pc_status st = wrap(pc::gen_rmat_batch(G, smin, smax, emin, emax, seed, &v), out);
        if (st == PC_OK) memcpy(voff, v.data(), v.size() * 8);
        return st;
    } catch (const std::bad_alloc&) {
        return fail(PC_ERR_OOM, "host allocation failed");
    }
}

pc_status pc_host_greedy_partition(const uint64_t* vlist, const int32_t* elist, uint64_t n, int32_t P, uint64_t seed,
                                   int32_t* v2p) {
    pc::clear_error();
    if (!vlist || (vlist[n] && !elist) || (n && !v2p)) return fail(PC_ERR_INVALID_INPUT, "null argument");
    if (P < 1) return fail(PC_ERR_INVALID_INPUT, "partition count must be positive");
    std::vector<int> out;
    pc::greedy_partition_host(n, vlist, elist, (size_t)P, seed, out);
    std::copy(out.begin(), out.end(), v2p);
    return PC_OK;
}

pc_status pc_synth_vertex_priority(uint64_t seed, uint64_t n, uint64_t* out) {
    pc::clear_error();
    if (n && !out) return fail(PC_ERR_INVALID_INPUT, "null output");
    const uint64_t key = pc_graph_key(seed, PC_GEN_PRIORITY);
    for (uint64_t v = 0; v < n; ++v) out[v] = pc_vertex_priority(key, (uint32_t)v);
    return PC_OK;
}

}  // extern "C"
