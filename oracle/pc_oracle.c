/*
 * TEST INFRASTRUCTURE -- the CPU oracle.  Only the tests, the smoke check and
 * bench.py's CPU-baseline leg may load this library; the product (libpc.so)
 * never does.
 *
 * A plain-C restatement of the reference algorithms of PartitionAndConquer
 * (src/Graph.cpp) on a symmetric CSR: n vertices, vlist[n+1] (uint64 offsets),
 * elist[m] (int32 ids, rows sorted ascending), weights[m] (int32).  Each
 * function names the reference lines it follows.  Parity of this restatement
 * is pinned against the reference itself, compiled here from its own sources
 * (oracle/_ref, see oracle/Makefile), through the fixtures in tests/golden/.
 */
#include "pc_oracle.h"

#include <limits.h>
#include <stdlib.h>
#include <string.h>

/* Graph::cnt_common_neis_less_than_merge (src/Graph.cpp:272-285). */
static uint64_t lt_merge(const uint64_t* vl, const int32_t* el, int64_t u, int64_t v, int32_t thr) {
    uint64_t up = vl[u], vp = vl[v], res = 0;
    while (up < vl[u + 1] && vp < vl[v + 1] && el[up] < thr && el[vp] < thr) {
        if (el[up] == el[vp]) { res++; up++; vp++; }
        else if (el[up] < el[vp]) up++;
        else vp++;
    }
    return res;
}

/* Graph::cnt_common_neis_merge (src/Graph.cpp:227-239). */
static uint64_t merge_cnt(const uint64_t* vl, const int32_t* el, int64_t u, int64_t v) {
    uint64_t up = vl[u], vp = vl[v], res = 0;
    while (up < vl[u + 1] && vp < vl[v + 1]) {
        if (el[up] == el[vp]) { res++; up++; vp++; }
        else if (el[up] < el[vp]) up++;
        else vp++;
    }
    return res;
}

/* |N(a) & N(b) & N(c)| by two sorted merges (the k-way
 * Graph::cnt_common_neis_merge(q), src/Graph.cpp:255-307, for k = 3). */
static uint64_t merge3(const uint64_t* vl, const int32_t* el, int32_t a, int32_t b, int32_t c) {
    uint64_t i = vl[a], ie = vl[a + 1], j = vl[b], je = vl[b + 1], k = vl[c], ke = vl[c + 1], res = 0;
    while (i < ie && j < je) {
        if (el[i] < el[j]) { i++; continue; }
        if (el[i] > el[j]) { j++; continue; }
        int32_t x = el[i];
        while (k < ke && el[k] < x) k++;
        if (k < ke && el[k] == x) res++;
        i++;
        j++;
    }
    return res;
}

/* Graph::solve_friend_triangle_merge (src/Graph.cpp:326-340) and the
 * partitioned forms (src/Graph.cpp:1222-1264, whose per-partition counts sum
 * to the whole-list count): positions j < k of nodes, the root skipped. */
uint64_t or_friend_triangle(uint64_t n, const uint64_t* vl, const int32_t* el, int32_t root, const int32_t* nodes,
                            uint64_t nn) {
    (void)n;
    uint64_t res = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : res)
    for (int64_t j = 0; j < (int64_t)nn; j++) {
        if (nodes[j] == root) continue;
        for (uint64_t k = (uint64_t)j + 1; k < nn; k++) {
            if (nodes[k] == root) continue;
            res += merge3(vl, el, root, nodes[j], nodes[k]);
        }
    }
    return res;
}

/* Partitioned_Graph::solve_square_counting (src/Graph.cpp:1291-1324): for
 * every u and v, w in N(u) with w < v < u, |N(v) & N(w) & [0, w)| (the
 * reference sums the partition-local counts, which add up to this). */
uint64_t or_square_count(uint64_t n, const uint64_t* vl, const int32_t* el) {
    uint64_t res = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : res)
    for (int64_t u = 0; u < (int64_t)n; u++) {
        for (uint64_t i = vl[u]; i < vl[u + 1]; i++) {
            int32_t v = el[i];
            if (v >= u) break;
            for (uint64_t j = vl[u]; j < vl[u + 1]; j++) {
                int32_t w = el[j];
                if (w >= v) break;
                res += lt_merge(vl, el, v, w, w);
            }
        }
    }
    return res;
}

/* Graph::solve_triangle_counting_merge (src/Graph.cpp:355-368). */
uint64_t or_tc_merge(uint64_t n, const uint64_t* vl, const int32_t* el) {
    uint64_t res = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : res)
    for (int64_t u = 0; u < (int64_t)n; u++) {
        for (uint64_t j = vl[u]; j < vl[u + 1]; j++) {
            int32_t v = el[j];
            if (u <= v) continue;
            res += lt_merge(vl, el, u, v, v);
        }
    }
    return res;
}

/* The loop of Graph::solve_triangle_counting_merge (src/Graph.cpp:358-365)
 * restricted to the given rows (a bounded sample for timing). */
uint64_t or_tc_rows(uint64_t n, const uint64_t* vl, const int32_t* el, const int32_t* rows, uint64_t nrows) {
    (void)n;
    uint64_t res = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : res)
    for (int64_t i = 0; i < (int64_t)nrows; i++) {
        int64_t u = rows[i];
        for (uint64_t j = vl[u]; j < vl[u + 1]; j++) {
            int32_t v = el[j];
            if (u <= v) continue;
            res += lt_merge(vl, el, u, v, v);
        }
    }
    return res;
}

/* Graph::solve_triangle_counting_galloping (src/Graph.cpp:342-353) with
 * Graph::cnt_common_neis_galloping (src/Graph.cpp:186-198): every ordered
 * edge, each element of the shorter list binary-searched in the longer. */
uint64_t or_tc_galloping(uint64_t n, const uint64_t* vl, const int32_t* el) {
    uint64_t res = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : res)
    for (int64_t u = 0; u < (int64_t)n; u++) {
        for (uint64_t j = vl[u]; j < vl[u + 1]; j++) {
            int64_t v = el[j];
            uint64_t us = vl[u], ue = vl[u + 1], vs = vl[v], ve = vl[v + 1];
            if (ue - us > ve - vs) { uint64_t t = us; us = vs; vs = t; t = ue; ue = ve; ve = t; }
            for (uint64_t i = us; i < ue; i++) {
                int32_t x = el[i];
                uint64_t lo = vs, hi = ve;
                while (lo < hi) {
                    uint64_t mid = lo + (hi - lo) / 2;
                    if (el[mid] < x) lo = mid + 1; else hi = mid;
                }
                if (lo < ve && el[lo] == x) res++;
            }
        }
    }
    return res;
}

/* Partitioned_Graph::Partitioned_Graph (src/Graph.cpp:1017-1069): for each
 * partition k (major), each vertex u, the sub-list N_k(u) = {v in N(u) :
 * v2p[v] == k} in the original order; out_vlist[k*n+u] is its start. */
int or_layout(uint64_t n, const uint64_t* vl, const int32_t* el, const int32_t* w, const int32_t* v2p, int32_t P,
              uint64_t* out_vl, int32_t* out_el, int32_t* out_w) {
    uint64_t pos = 0;
    for (int32_t k = 0; k < P; k++) {
        for (uint64_t u = 0; u < n; u++) {
            out_vl[(uint64_t)k * n + u] = pos;
            for (uint64_t j = vl[u]; j < vl[u + 1]; j++) {
                if (v2p[el[j]] != k) continue;
                out_el[pos] = el[j];
                if (w && out_w) out_w[pos] = w[j];
                pos++;
            }
        }
    }
    out_vl[(uint64_t)P * n] = pos;
    return 0;
}

/* Partitioned_Graph::solve_triangle_counting_merge (src/Graph.cpp:1346-1362)
 * on the layout above, with cnt_common_neis_less_than_merge
 * (src/Graph.cpp:1132-1153). */
uint64_t or_tc_partitioned(uint64_t n, const uint64_t* pvl, const int32_t* pel, int32_t P) {
    uint64_t res = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : res)
    for (int32_t i = 0; i < P; i++) {
        for (int32_t j = 0; j < P; j++) {
            for (uint64_t u = 0; u < n; u++) {
                for (uint64_t k = pvl[(uint64_t)j * n + u]; k < pvl[(uint64_t)j * n + u + 1]; k++) {
                    int32_t v = pel[k];
                    if ((uint64_t)v >= u) break;
                    uint64_t up = pvl[(uint64_t)i * n + u], ue = pvl[(uint64_t)i * n + u + 1];
                    uint64_t vp = pvl[(uint64_t)i * n + v], ve = pvl[(uint64_t)i * n + v + 1];
                    while (up < ue && vp < ve && pel[up] < v && pel[vp] < v) {
                        if (pel[up] < pel[vp]) up++;
                        else if (pel[up] > pel[vp]) vp++;
                        else { res++; up++; vp++; }
                    }
                }
            }
        }
    }
    return res;
}

/* Graph::solve_lcc_merge (src/Graph.cpp:828-840). */
void or_lcc(uint64_t n, const uint64_t* vl, const int32_t* el, double* out) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t u = 0; u < (int64_t)n; u++) {
        uint64_t d = vl[u + 1] - vl[u];
        out[u] = 0.0;
        if (d < 1) continue;
        double s = 0.0;
        for (uint64_t j = vl[u]; j < vl[u + 1]; j++) s += (double)merge_cnt(vl, el, u, el[j]);
        out[u] = s / (double)(d * (d - 1));
    }
}

/* Graph::solve_jsim_merge's formula (src/Graph.cpp:806-809) for every CSR
 * entry (u, v), rounded to fp32. */
void or_jaccard_edges(uint64_t n, const uint64_t* vl, const int32_t* el, float* out) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t u = 0; u < (int64_t)n; u++) {
        uint64_t du = vl[u + 1] - vl[u];
        for (uint64_t j = vl[u]; j < vl[u + 1]; j++) {
            int32_t v = el[j];
            uint64_t dv = vl[v + 1] - vl[v];
            double c = (double)merge_cnt(vl, el, u, v);
            out[j] = (float)(c / ((double)(du + dv) - c));
        }
    }
}

/* or_jaccard_edges restricted to the rows listed (a bounded exact sample of a
 * graph too large for the full sweep): out holds, row after row in the order
 * given, one value per entry of each row. */
void or_jaccard_rows(uint64_t n, const uint64_t* vl, const int32_t* el, const int32_t* rows, uint64_t nrows,
                     float* out) {
    (void)n;
    uint64_t* base = malloc((nrows + 1) * sizeof(uint64_t));
    base[0] = 0;
    for (uint64_t i = 0; i < nrows; i++) base[i + 1] = base[i] + (vl[rows[i] + 1] - vl[rows[i]]);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < (int64_t)nrows; i++) {
        int64_t u = rows[i];
        uint64_t du = vl[u + 1] - vl[u];
        for (uint64_t j = vl[u]; j < vl[u + 1]; j++) {
            int32_t v = el[j];
            uint64_t dv = vl[v + 1] - vl[v];
            double c = (double)merge_cnt(vl, el, u, v);
            out[base[i] + (j - vl[u])] = (float)(c / ((double)(du + dv) - c));
        }
    }
    free(base);
}

/* A size-independent audit of an all-edge Jaccard result J[m] (the
 * Graph::solve_jsim_merge formula per CSR entry, stored as float).  Per entry
 * (u, v) with D = d(u) + d(v), the common-neighbour count c is recovered as
 * round(J D / (1 + J)), and the entry must round-trip: (float)(c / (D - c))
 * == J bit for bit (adjacent c give distinct floats while D < 2^24).  The
 * twin entry (v, u), found by binary search in N(v), must hold the same
 * value.  *sum_c is the sum of c over all entries, which is 6 T for a graph
 * with T triangles (each triangle lies on three edges, each stored twice). */
void or_jaccard_audit(uint64_t n, const uint64_t* vl, const int32_t* el, const float* J, uint64_t* sum_c,
                      uint64_t* bad_roundtrip, uint64_t* bad_twin) {
    uint64_t sc = 0, br = 0, bt = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : sc, br, bt)
    for (int64_t u = 0; u < (int64_t)n; u++) {
        uint64_t du = vl[u + 1] - vl[u];
        for (uint64_t j = vl[u]; j < vl[u + 1]; j++) {
            int32_t v = el[j];
            uint64_t D = du + (vl[v + 1] - vl[v]);
            double x = (double)J[j];
            double cr = x * (double)D / (1.0 + x);
            int64_t c = (int64_t)(cr + 0.5);
            if (c < 0 || (uint64_t)c > D / 2 || (float)((double)c / ((double)D - (double)c)) != J[j]) br++;
            else sc += (uint64_t)c;
            uint64_t lo = vl[v], hi = vl[v + 1];
            while (lo < hi) {
                uint64_t mid = (lo + hi) >> 1;
                if (el[mid] < (int32_t)u) lo = mid + 1; else hi = mid;
            }
            if (lo == vl[v + 1] || el[lo] != (int32_t)u || J[lo] != J[j]) bt++;
        }
    }
    *sum_c = sc;
    *bad_roundtrip = br;
    *bad_twin = bt;
}

/* Graph::solve_jsim_merge (src/Graph.cpp:798-812). */
void or_jaccard_queries(uint64_t n, const uint64_t* vl, const int32_t* el, const int32_t* q, int32_t nq, double* out) {
    (void)n;
    for (int32_t i = 0; i < nq; i++) {
        uint64_t du = vl[q[i] + 1] - vl[q[i]];
        for (int32_t j = 0; j < nq; j++) {
            uint64_t dv = vl[q[j] + 1] - vl[q[j]];
            double c = (double)merge_cnt(vl, el, q[i], q[j]);
            out[(int64_t)i * nq + j] = c / ((double)(du + dv) - c);
        }
    }
}

/* Graph::batch_cnt_common_neis_merge over pairs (src/Graph.cpp:431-438). */
void or_batch_pairs(uint64_t n, const uint64_t* vl, const int32_t* el, const int32_t* pairs, uint64_t nq, uint64_t* out) {
    (void)n;
    for (uint64_t i = 0; i < nq; i++) out[i] = merge_cnt(vl, el, pairs[2 * i], pairs[2 * i + 1]);
}

/* Graph::cnt_common_neis_merge(q) (src/Graph.cpp:255-270) per k-set. */
void or_batch_sets(uint64_t n, const uint64_t* vl, const int32_t* el, const int32_t* ids, const uint64_t* offs,
                   uint64_t nq, uint64_t* out) {
    (void)n;
    for (uint64_t i = 0; i < nq; i++) {
        const int32_t* q = ids + offs[i];
        uint64_t k = offs[i + 1] - offs[i];
        int32_t q0 = q[0];
        uint64_t cap = vl[q0 + 1] - vl[q0];
        int32_t* cur = (int32_t*)malloc((cap + 1) * sizeof(int32_t));
        int32_t* nxt = (int32_t*)malloc((cap + 1) * sizeof(int32_t));
        uint64_t nc = cap;
        memcpy(cur, el + vl[q0], cap * sizeof(int32_t));
        for (uint64_t t = 1; t + 1 < k; t++) {
            uint64_t a = vl[q[t]], ae = vl[q[t] + 1], b = 0, nn = 0;
            while (a < ae && b < nc) {
                if (el[a] == cur[b]) { nxt[nn++] = cur[b]; a++; b++; }
                else if (el[a] < cur[b]) a++;
                else b++;
            }
            int32_t* tmp = cur; cur = nxt; nxt = tmp; nc = nn;
        }
        int32_t ql = q[k - 1];
        uint64_t a = vl[ql], ae = vl[ql + 1], b = 0, res = 0;
        while (a < ae && b < nc) {
            if (el[a] == cur[b]) { res++; a++; b++; }
            else if (el[a] < cur[b]) a++;
            else b++;
        }
        out[i] = res;
        free(cur);
        free(nxt);
    }
}

/* BFS depth from src (the level structure of Graph::solve_bfs,
 * src/Graph.cpp:621-646) in Partitioned_Graph::solve_bfs's output convention
 * (src/Graph.cpp:1702-1741): rank[src] = -1, level r >= 1, unreached INT_MAX. */
void or_bfs(uint64_t n, const uint64_t* vl, const int32_t* el, int32_t src, int32_t* rank) {
    int32_t* q = (int32_t*)malloc((n + 1) * sizeof(int32_t));
    for (uint64_t u = 0; u < n; u++) rank[u] = INT_MAX;
    rank[src] = -1;
    uint64_t head = 0, tail = 0;
    q[tail++] = src;
    int32_t level = 0;
    while (head < tail) {
        uint64_t end = tail;
        level++;
        for (; head < end; head++) {
            int32_t u = q[head];
            for (uint64_t j = vl[u]; j < vl[u + 1]; j++) {
                int32_t v = el[j];
                if (rank[v] == INT_MAX) { rank[v] = level; q[tail++] = v; }
            }
        }
    }
    free(q);
}

/* Graph::solve_sssp (src/Graph.cpp:842-868): Dijkstra with a binary heap of
 * (distance, vertex) entries and lazy deletion; unreached = INT_MAX / 2. */
typedef struct { int64_t d; int32_t v; } HeapItem;
static void heap_push(HeapItem* h, uint64_t* sz, HeapItem x) {
    uint64_t i = (*sz)++;
    while (i > 0) {
        uint64_t p = (i - 1) / 2;
        if (h[p].d <= x.d) break;
        h[i] = h[p];
        i = p;
    }
    h[i] = x;
}
static HeapItem heap_pop(HeapItem* h, uint64_t* sz) {
    HeapItem top = h[0], x = h[--(*sz)];
    uint64_t i = 0;
    for (;;) {
        uint64_t l = 2 * i + 1, r = l + 1, s = i;
        int64_t sd = x.d;
        if (l < *sz && h[l].d < sd) { s = l; sd = h[l].d; }
        if (r < *sz && h[r].d < sd) { s = r; }
        if (s == i) break;
        h[i] = h[s];
        i = s;
    }
    if (*sz) h[i] = x;
    return top;
}
void or_sssp(uint64_t n, const uint64_t* vl, const int32_t* el, const int32_t* w, int32_t src, int32_t* dist) {
    for (uint64_t u = 0; u < n; u++) dist[u] = INT_MAX / 2;
    uint64_t m = vl[n];
    HeapItem* h = (HeapItem*)malloc((m + 2) * sizeof(HeapItem));
    uint8_t* done = (uint8_t*)calloc(n + 1, 1);
    uint64_t sz = 0;
    dist[src] = 0;
    HeapItem s0 = {0, src};
    heap_push(h, &sz, s0);
    while (sz) {
        HeapItem t = heap_pop(h, &sz);
        int32_t u = t.v;
        if (done[u]) continue;
        done[u] = 1;
        for (uint64_t j = vl[u]; j < vl[u + 1]; j++) {
            int32_t v = el[j];
            int64_t nd = (int64_t)dist[u] + w[j];
            if (dist[v] > nd) {
                dist[v] = (int32_t)nd;
                HeapItem x = {nd, v};
                heap_push(h, &sz, x);
            }
        }
    }
    free(h);
    free(done);
}

/* Partitioned_Graph::page_rank's recurrence (src/Graph.cpp:1563-1596) in
 * FP64: degs = d / damping, x0 = degs / n; per iteration x[u] /= degs[u],
 * new[v] = (1 - damping) / n + sum_{u in N(v)} x[u] (ascending u).  With
 * init != NULL, x0 = init: Graph::page_rank (src/Graph.cpp:534-554), whose
 * iteration is the same recurrence. */
void or_pagerank_f64(uint64_t n, const uint64_t* vl, const int32_t* el, double damping, int32_t iters,
                     const double* init, double* out) {
    double* degs = (double*)malloc((n + 1) * sizeof(double));
    double* x = (double*)malloc((n + 1) * sizeof(double));
    const double base = (1.0 - damping) / (double)n;
    for (uint64_t u = 0; u < n; u++) {
        degs[u] = (double)(vl[u + 1] - vl[u]) / damping;
        x[u] = init ? init[u] : degs[u] / (double)n;
    }
    for (int32_t it = 0; it < iters; it++) {
        for (uint64_t u = 0; u < n; u++) x[u] = degs[u] > 0 ? x[u] / degs[u] : 0.0;
        for (uint64_t v = 0; v < n; v++) {
            double s = base;
            for (uint64_t j = vl[v]; j < vl[v + 1]; j++) s += x[el[j]];
            out[v] = s;
        }
        memcpy(x, out, n * sizeof(double));
    }
    if (iters <= 0) memcpy(out, x, n * sizeof(double));
    free(degs);
    free(x);
}

/* Core numbers as Graph::solve_kcore peels them (src/Graph.cpp:662-719): a
 * vertex removed while peeling level k (degree < k) has core number k - 1,
 * for levels k < n.
 * Computed with the O(m) bucket order of Batagelj & Zaversnik (2003), which
 * yields the same numbers. */
int32_t or_kcore(uint64_t n, const uint64_t* vl, const int32_t* el, int32_t* core) {
    if (n == 0) return 0;
    int32_t* deg = (int32_t*)malloc(n * sizeof(int32_t));
    int32_t md = 0;
    for (uint64_t u = 0; u < n; u++) {
        deg[u] = (int32_t)(vl[u + 1] - vl[u]);
        if (deg[u] > md) md = deg[u];
    }
    int64_t* bin = (int64_t*)calloc((size_t)md + 2, sizeof(int64_t));
    int64_t* pos = (int64_t*)malloc(n * sizeof(int64_t));
    int32_t* vert = (int32_t*)malloc(n * sizeof(int32_t));
    for (uint64_t u = 0; u < n; u++) bin[deg[u]]++;
    int64_t start = 0;
    for (int32_t d = 0; d <= md; d++) { int64_t c = bin[d]; bin[d] = start; start += c; }
    for (uint64_t u = 0; u < n; u++) { pos[u] = bin[deg[u]]; vert[pos[u]] = (int32_t)u; bin[deg[u]]++; }
    for (int32_t d = md; d >= 1; d--) bin[d] = bin[d - 1];
    bin[0] = 0;
    int32_t largest = 0;
    for (uint64_t i = 0; i < n; i++) {
        int32_t v = vert[i];
        core[v] = deg[v];
        if (deg[v] > largest) largest = deg[v];
        for (uint64_t j = vl[v]; j < vl[v + 1]; j++) {
            int32_t u = el[j];
            if (deg[u] > deg[v]) {
                int32_t du = deg[u];
                int64_t pu = pos[u], pw = bin[du];
                int32_t w = vert[pw];
                if (u != w) { pos[u] = pw; vert[pu] = w; pos[w] = pu; vert[pw] = u; }
                bin[du]++;
                deg[u]--;
            }
        }
    }
    free(deg); free(bin); free(pos); free(vert);
    /* The reference peels levels k = 1 .. n-1 only (src/Graph.cpp:683): a
     * vertex still present after level n-1 keeps its initial 0.  That happens
     * exactly when the graph is complete (core number n-1 everywhere). */
    if (n >= 2 && largest >= (int32_t)n - 1) {
        largest = 0;
        for (uint64_t u = 0; u < n; u++) {
            if (core[u] >= (int32_t)n - 1) core[u] = 0;
            if (core[u] > largest) largest = core[u];
        }
    }
    return largest;
}

/* The maximal independent set Graph::solve_mis computes (src/Graph.cpp:721-780):
 * a vertex joins once every smaller-id neighbour is out, i.e. the
 * lexicographically-first MIS in id order. */
void or_mis(uint64_t n, const uint64_t* vl, const int32_t* el, int32_t* res) {
    for (uint64_t u = 0; u < n; u++) {
        int in = 1;
        for (uint64_t j = vl[u]; j < vl[u + 1]; j++) {
            int32_t v = el[j];
            if ((uint64_t)v >= u) break; /* rows are sorted */
            if (res[v]) { in = 0; break; }
        }
        res[u] = in;
    }
}

/* The same greedy rule in ascending (priority[u], u) order instead of id
 * order: the reference run on ids relabelled by that order, mapped back. */
static const uint64_t* g_prio;
static int cmp_prio(const void* a, const void* b) {
    int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    if (g_prio[x] != g_prio[y]) return g_prio[x] < g_prio[y] ? -1 : 1;
    return (x > y) - (x < y);
}
void or_mis_priority(uint64_t n, const uint64_t* vl, const int32_t* el, const uint64_t* priority, int32_t* res) {
    int32_t* order = (int32_t*)malloc((n + 1) * sizeof(int32_t));
    for (uint64_t u = 0; u < n; u++) { order[u] = (int32_t)u; res[u] = 0; }
    g_prio = priority;
    qsort(order, n, sizeof(int32_t), cmp_prio);
    for (uint64_t i = 0; i < n; i++) {
        int32_t u = order[i];
        int in = 1;
        for (uint64_t j = vl[u]; j < vl[u + 1]; j++) {
            int32_t v = el[j];
            if (res[v]) { in = 0; break; }
        }
        res[u] = in;
    }
    free(order);
}

/* Graph::solve_cdlp (src/Graph.cpp:648-660): labels[u] <- max over N(u) of
 * labels[v], 0 for isolated u, `iters` times. */
void or_cdlp(uint64_t n, const uint64_t* vl, const int32_t* el, int32_t iters, int32_t* labels) {
    int32_t* tmp = (int32_t*)malloc((n + 1) * sizeof(int32_t));
    for (int32_t it = 0; it < iters; it++) {
        for (uint64_t u = 0; u < n; u++) {
            int32_t t = 0;
            for (uint64_t j = vl[u]; j < vl[u + 1]; j++)
                if (labels[el[j]] > t) t = labels[el[j]];
            tmp[u] = t;
        }
        memcpy(labels, tmp, n * sizeof(int32_t));
    }
    free(tmp);
}
