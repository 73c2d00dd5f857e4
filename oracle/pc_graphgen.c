/*
 * TEST INFRASTRUCTURE -- seeded synthetic graphs for the CPU side of the
 * checks, so that the reference arm of the benchmark and the pinned-count
 * script build their inputs without loading the product library.
 *
 * An independent restatement of the graph generators the product uses
 * (counter-based draws, RMAT / Erdos-Renyi / Chung-Lu edge streams,
 * symmetrise + drop self-loops + deduplicate + sort, relabel by descending
 * degree with ties by id), written from their published definitions:
 *   - draws: the SplitMix64 output function (Steele, Lea, Flood, OOPSLA 2014)
 *     applied to key + counter * golden gamma; a graph's key mixes its seed
 *     and generator kind;
 *   - RMAT: Chakrabarti, Zhan, Faloutsos (SDM 2004), (a,b,c,d) =
 *     (0.57,0.19,0.19,0.05) compared as 32-bit fixed-point thresholds, two
 *     levels per 64-bit draw, most significant bit first;
 *   - Chung-Lu: expected degrees w_i = (i + i0)^(-1/(beta-1)), i0 bisected so
 *     that vertex 0 expects dmax, endpoints by inverse CDF over a 2^62 table.
 * The test suite checks that these arrays equal the product's host and
 * device generators bit for bit, so a graph named by (kind, scale, edges,
 * seed) is the same on both sides.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <omp.h>

typedef struct og_graph {
    uint64_t n, m;
    uint64_t* vl;
    int32_t* el;
} og_graph;

/* ---- draws -------------------------------------------------------------------- */

static const uint64_t kGamma = 0x9E3779B97F4A7C15ULL;

static inline uint64_t sm_out(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

enum { KIND_RMAT = 1, KIND_ER = 2, KIND_CHUNG_LU = 3, KIND_BATCH = 6 };

static inline uint64_t key_of(uint64_t seed, uint64_t kind) {
    return sm_out(sm_out(seed * kGamma + 0x632BE59BD9B4E019ULL) ^ (kind * 0xD1B54A32D192ED03ULL));
}

static inline uint64_t draw(uint64_t key, uint64_t ctr) { return sm_out(key + ctr * kGamma); }

/* ---- edge streams ---------------------------------------------------------------- */

static void rmat_stream(uint32_t scale, uint64_t ne, uint64_t seed, uint32_t* s, uint32_t* d) {
    const uint64_t key = key_of(seed, KIND_RMAT);
    /* floor(p * 2^32) for the cumulative quadrant probabilities 0.57, 0.76, 0.95 */
    const uint32_t tA = 2448131358u, tAB = 3264175144u, tABC = 4080218931u;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < (int64_t)ne; k++) {
        uint32_t u = 0, v = 0;
        uint64_t x = 0;
        for (uint32_t lvl = 0; lvl < scale; lvl++) {
            if ((lvl & 1) == 0) x = draw(key, ((uint64_t)k << 5) | (lvl >> 1));
            uint32_t r = (uint32_t)(x >> (32 * (lvl & 1)));
            uint32_t bit = 1u << (scale - 1 - lvl);
            if (r >= tABC) { u |= bit; v |= bit; }
            else if (r >= tAB) u |= bit;
            else if (r >= tA) v |= bit;
        }
        s[k] = u;
        d[k] = v;
    }
}

static void er_stream(uint32_t scale, uint64_t ne, uint64_t seed, uint32_t* s, uint32_t* d) {
    const uint64_t key = key_of(seed, KIND_ER);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < (int64_t)ne; k++) {
        uint64_t x = draw(key, (uint64_t)k);
        s[k] = (uint32_t)(x >> (64 - scale));
        d[k] = (uint32_t)((x & 0xFFFFFFFFull) >> (32 - scale));
    }
}

static double cl_expected_max(uint64_t n, uint64_t ne, double alpha, double i0) {
    double sum = 0.0;
    for (uint64_t i = 0; i < n; i++) sum += pow((double)i + i0, -alpha);
    return 2.0 * (double)ne * pow(i0, -alpha) / sum;
}

static int chung_lu_stream(uint32_t scale, uint64_t ne, double beta, uint64_t dmax, uint64_t seed, uint32_t* s,
                           uint32_t* d) {
    const uint64_t n = 1ull << scale;
    const double alpha = 1.0 / (beta - 1.0);
    double lo = 1e-3, hi = (double)n;
    for (int it = 0; it < 60; it++) {
        double mid = sqrt(lo * hi);
        if (cl_expected_max(n, ne, alpha, mid) > (double)dmax) lo = mid; else hi = mid;
    }
    const double i0 = hi;
    double* w = malloc(n * sizeof(double));
    uint64_t* cdf = malloc(n * sizeof(uint64_t));
    if (!w || !cdf) { free(w); free(cdf); return -1; }
    double tot = 0.0, acc = 0.0;
    for (uint64_t i = 0; i < n; i++) { w[i] = pow((double)i + i0, -alpha); tot += w[i]; }
    const double two62 = 4611686018427387904.0;
    for (uint64_t i = 0; i < n; i++) {
        acc += w[i];
        double f = floor(acc / tot * two62);
        cdf[i] = (uint64_t)(f < two62 ? f : two62);
    }
    cdf[n - 1] = (uint64_t)two62;
    free(w);
    const uint64_t key = key_of(seed, KIND_CHUNG_LU);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < (int64_t)ne; k++) {
        for (int e = 0; e < 2; e++) {
            uint64_t r = draw(key, ((uint64_t)k << 1) | (uint64_t)e) >> 2;
            /* first index whose cdf exceeds r */
            uint64_t a = 0, b = n;
            while (a < b) {
                uint64_t mid = (a + b) >> 1;
                if (cdf[mid] <= r) a = mid + 1; else b = mid;
            }
            uint32_t idx = (uint32_t)(a < n ? a : n - 1);
            if (e) d[k] = idx; else s[k] = idx;
        }
    }
    free(cdf);
    return 0;
}

/* ---- CSR building ------------------------------------------------------------------ */

static int cmp_i32(const void* x, const void* y) {
    int32_t a = *(const int32_t*)x, b = *(const int32_t*)y;
    return (a > b) - (a < b);
}

/* Sorts a[0..len) ascending: insertion sort for short rows, qsort for medium
 * ones, two 16-bit LSD counting passes through tmp for rows of 2^16 ids and
 * more (ids are non-negative int32). */
static void sort_ids(int32_t* a, uint64_t len, int32_t* tmp) {
    if (len <= 32) {
        for (uint64_t i = 1; i < len; i++) {
            int32_t x = a[i];
            uint64_t j = i;
            while (j > 0 && a[j - 1] > x) { a[j] = a[j - 1]; j--; }
            a[j] = x;
        }
        return;
    }
    if (len < (1u << 16)) {
        qsort(a, len, sizeof(int32_t), cmp_i32);
        return;
    }
    enum { R = 1 << 16 };
    uint64_t* cnt = malloc(R * sizeof(uint64_t));
    for (int pass = 0; pass < 2; pass++) {
        int32_t* src = pass ? tmp : a;
        int32_t* dst = pass ? a : tmp;
        const int sh = 16 * pass;
        memset(cnt, 0, R * sizeof(uint64_t));
        for (uint64_t i = 0; i < len; i++) cnt[((uint32_t)src[i] >> sh) & 0xFFFF]++;
        uint64_t run = 0;
        for (int b = 0; b < R; b++) { uint64_t c = cnt[b]; cnt[b] = run; run += c; }
        for (uint64_t i = 0; i < len; i++) dst[cnt[((uint32_t)src[i] >> sh) & 0xFFFF]++] = src[i];
    }
    free(cnt);
}

static void scan(const uint64_t* cnt, uint64_t n, uint64_t* off) {
    uint64_t s = 0;
    for (uint64_t i = 0; i < n; i++) { off[i] = s; s += cnt[i]; }
    off[n] = s;
}

static uint64_t max_row(const uint64_t* off, uint64_t n) {
    uint64_t mx = 0;
#pragma omp parallel for reduction(max : mx)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        uint64_t d = off[i + 1] - off[i];
        if (d > mx) mx = d;
    }
    return mx;
}

/* Symmetric CSR of the edge stream: both directions, self-loops dropped,
 * duplicates removed, rows ascending. */
static og_graph* build_csr(uint64_t n, uint64_t ne, const uint32_t* s, const uint32_t* d) {
    uint64_t* deg = calloc(n, sizeof(uint64_t));
    uint64_t* off = malloc((n + 1) * sizeof(uint64_t));
    if (!deg || !off) { free(deg); free(off); return NULL; }
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < (int64_t)ne; k++) {
        if (s[k] == d[k]) continue;
        __atomic_fetch_add(&deg[s[k]], 1, __ATOMIC_RELAXED);
        __atomic_fetch_add(&deg[d[k]], 1, __ATOMIC_RELAXED);
    }
    scan(deg, n, off);
    int32_t* col = malloc((off[n] ? off[n] : 1) * sizeof(int32_t));
    if (!col) { free(deg); free(off); return NULL; }
    memset(deg, 0, n * sizeof(uint64_t));
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < (int64_t)ne; k++) {
        uint32_t u = s[k], v = d[k];
        if (u == v) continue;
        col[off[u] + __atomic_fetch_add(&deg[u], 1, __ATOMIC_RELAXED)] = (int32_t)v;
        col[off[v] + __atomic_fetch_add(&deg[v], 1, __ATOMIC_RELAXED)] = (int32_t)u;
    }
    const uint64_t mx = max_row(off, n);
#pragma omp parallel
    {
        int32_t* tmp = malloc((mx ? mx : 1) * sizeof(int32_t));
#pragma omp for schedule(dynamic, 1024)
        for (int64_t i = 0; i < (int64_t)n; i++) {
            int32_t* a = col + off[i];
            uint64_t len = off[i + 1] - off[i], u = 0;
            sort_ids(a, len, tmp);
            for (uint64_t j = 0; j < len; j++)
                if (u == 0 || a[j] != a[u - 1]) a[u++] = a[j];
            deg[i] = u;
        }
        free(tmp);
    }
    og_graph* g = calloc(1, sizeof(og_graph));
    g->n = n;
    g->vl = malloc((n + 1) * sizeof(uint64_t));
    scan(deg, n, g->vl);
    g->m = g->vl[n];
    g->el = malloc((g->m ? g->m : 1) * sizeof(int32_t));
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < (int64_t)n; i++) memcpy(g->el + g->vl[i], col + off[i], deg[i] * sizeof(int32_t));
    free(col);
    free(off);
    free(deg);
    return g;
}

/* New ids by descending degree, ties by ascending id (a counting sort by
 * degree visiting ids in ascending order); rows mapped and re-sorted. */
static og_graph* relabel_by_degree(og_graph* g) {
    const uint64_t n = g->n;
    uint64_t mx = max_row(g->vl, n);
    uint64_t* start = calloc(mx + 2, sizeof(uint64_t));
    int32_t* old2new = malloc(n * sizeof(int32_t));
    int32_t* new2old = malloc(n * sizeof(int32_t));
    for (uint64_t i = 0; i < n; i++) start[mx - (g->vl[i + 1] - g->vl[i])]++;
    uint64_t run = 0;
    for (uint64_t b = 0; b <= mx; b++) { uint64_t c = start[b]; start[b] = run; run += c; }
    for (uint64_t i = 0; i < n; i++) {
        uint64_t r = start[mx - (g->vl[i + 1] - g->vl[i])]++;
        old2new[i] = (int32_t)r;
        new2old[r] = (int32_t)i;
    }
    free(start);
    og_graph* r = calloc(1, sizeof(og_graph));
    r->n = n;
    r->m = g->m;
    r->vl = malloc((n + 1) * sizeof(uint64_t));
    r->el = malloc((g->m ? g->m : 1) * sizeof(int32_t));
    uint64_t s = 0;
    for (uint64_t i = 0; i < n; i++) {
        r->vl[i] = s;
        s += g->vl[new2old[i] + 1] - g->vl[new2old[i]];
    }
    r->vl[n] = s;
#pragma omp parallel
    {
        int32_t* tmp = malloc((mx ? mx : 1) * sizeof(int32_t));
#pragma omp for schedule(dynamic, 1024)
        for (int64_t i = 0; i < (int64_t)n; i++) {
            const int32_t o = new2old[i];
            const uint64_t b = g->vl[o], len = g->vl[o + 1] - b;
            int32_t* dst = r->el + r->vl[i];
            for (uint64_t k = 0; k < len; k++) dst[k] = old2new[g->el[b + k]];
            sort_ids(dst, len, tmp);
        }
        free(tmp);
    }
    free(old2new);
    free(new2old);
    return r;
}

static void og_release(og_graph* g) {
    if (!g) return;
    free(g->vl);
    free(g->el);
    free(g);
}

static og_graph* finish(uint64_t n, uint64_t ne, uint32_t* s, uint32_t* d, int relabel) {
    og_graph* g = build_csr(n, ne, s, d);
    free(s);
    free(d);
    if (!g || !relabel) return g;
    og_graph* r = relabel_by_degree(g);
    og_release(g);
    return r;
}

/* ---- entry points ---------------------------------------------------------------- */

og_graph* og_rmat(uint32_t scale, uint64_t edge_factor, uint64_t seed, int relabel) {
    const uint64_t n = 1ull << scale, ne = n * edge_factor;
    uint32_t* s = malloc(ne * sizeof(uint32_t));
    uint32_t* d = malloc(ne * sizeof(uint32_t));
    if (!s || !d) { free(s); free(d); return NULL; }
    rmat_stream(scale, ne, seed, s, d);
    return finish(n, ne, s, d, relabel);
}

og_graph* og_er(uint32_t scale, uint64_t nedges, uint64_t seed, int relabel) {
    uint32_t* s = malloc(nedges * sizeof(uint32_t));
    uint32_t* d = malloc(nedges * sizeof(uint32_t));
    if (!s || !d) { free(s); free(d); return NULL; }
    er_stream(scale, nedges, seed, s, d);
    return finish(1ull << scale, nedges, s, d, relabel);
}

og_graph* og_chung_lu(uint32_t scale, uint64_t nedges, double beta, uint64_t dmax, uint64_t seed, int relabel) {
    uint32_t* s = malloc(nedges * sizeof(uint32_t));
    uint32_t* d = malloc(nedges * sizeof(uint32_t));
    if (!s || !d || chung_lu_stream(scale, nedges, beta, dmax, seed, s, d)) { free(s); free(d); return NULL; }
    return finish(1ull << scale, nedges, s, d, relabel);
}

/* The batch arena: graph g has scale smin + draw(2g) mod (smax-smin+1) and
 * edge factor emin + draw(2g+1) mod (emax-emin+1) under the batch key, is the
 * degree-relabelled RMAT graph of seed g, and owns the arena ids
 * [voff[g], voff[g+1]); voff must hold G+1 entries. */
og_graph* og_rmat_batch(uint32_t G, uint32_t smin, uint32_t smax, uint32_t emin, uint32_t emax, uint64_t seed,
                        uint64_t* voff) {
    const uint64_t key = key_of(seed, KIND_BATCH);
    og_graph** gs = calloc(G, sizeof(og_graph*));
    for (uint32_t g = 0; g < G; g++) {
        uint32_t sc = smin + (uint32_t)(draw(key, 2 * (uint64_t)g) % (uint64_t)(smax - smin + 1));
        uint32_t ef = emin + (uint32_t)(draw(key, 2 * (uint64_t)g + 1) % (uint64_t)(emax - emin + 1));
        gs[g] = og_rmat(sc, ef, g, 1);
    }
    og_graph* a = calloc(1, sizeof(og_graph));
    voff[0] = 0;
    uint64_t m = 0;
    for (uint32_t g = 0; g < G; g++) {
        voff[g + 1] = voff[g] + gs[g]->n;
        m += gs[g]->m;
    }
    a->n = voff[G];
    a->m = m;
    a->vl = malloc((a->n + 1) * sizeof(uint64_t));
    a->el = malloc((m ? m : 1) * sizeof(int32_t));
    uint64_t eb = 0;
    for (uint32_t g = 0; g < G; g++) {
        const og_graph* x = gs[g];
        for (uint64_t u = 0; u < x->n; u++) a->vl[voff[g] + u] = eb + x->vl[u];
        for (uint64_t k = 0; k < x->m; k++) a->el[eb + k] = x->el[k] + (int32_t)voff[g];
        eb += x->m;
        og_release(gs[g]);
    }
    a->vl[a->n] = m;
    free(gs);
    return a;
}

uint64_t og_n(const og_graph* g) { return g->n; }
uint64_t og_m(const og_graph* g) { return g->m; }

void og_copy(const og_graph* g, uint64_t* vl, int32_t* el) {
    memcpy(vl, g->vl, (g->n + 1) * sizeof(uint64_t));
    memcpy(el, g->el, g->m * sizeof(int32_t));
}

void og_free(og_graph* g) { og_release(g); }
