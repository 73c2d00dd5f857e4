/*
 * pc.h -- C ABI of the B200 partitioned-CSR analytics library (libpc.so).
 *
 * This is the drop-in boundary for the hot path of PartitionAndConquer: the
 * `Graph` / `Partitioned_Graph` classes of the reference (src/Graph.hpp:38-155).
 * Every entry point below names the reference member it replaces.  The
 * reference has no FFI of its own; its only caller is the CLI driver
 * (src/test.cpp:86-390), and the C++ host classes in pc_graph.hpp forward to
 * these functions.
 *
 * Conventions
 *  - Plain C types only: pointers and sizes.  Vertex ids are int32 (VID,
 *    src/Graph.hpp:23), edge offsets uint64 (EID, src/Graph.hpp:24), weights
 *    int32 (src/Graph.hpp:25).
 *  - Input and output arrays are HOST memory owned by the caller, unless a
 *    function says otherwise.  Device memory is owned by the handles.
 *  - Every call is synchronous (as the reference's member functions are) and
 *    returns a pc_status.  On failure pc_last_error() returns a message for
 *    the calling thread.
 *  - One CUDA stream per graph handle; a handle must not be used from two
 *    host threads at once.
 *  - There is no CPU fallback: without a usable CUDA device every compute
 *    call returns PC_ERR_CUDA (or PC_ERR_NO_DEVICE).
 */
#ifndef PC_H
#define PC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PC_OK = 0,
    PC_ERR_INVALID_INPUT = 1, /* malformed CSR / partition vector / argument */
    PC_ERR_OOM = 2,           /* device or pinned-host allocation failed */
    PC_ERR_CUDA = 3,          /* a CUDA runtime call failed */
    PC_ERR_TIMEOUT = 4,       /* a bounded device-side wait gave up */
    PC_ERR_NO_DEVICE = 5,     /* no CUDA device is visible */
    PC_ERR_UNSUPPORTED = 6    /* option not available for this handle */
} pc_status;

typedef struct pc_graph pc_graph;   /* device-resident symmetric CSR */
typedef struct pc_pgraph pc_pgraph; /* partitioned view of a pc_graph */

/* ---- library ---------------------------------------------------------- */

/* Message of the last failed call on this thread ("" if none). */
const char* pc_last_error(void);
/* Library version string. */
const char* pc_version(void);
/* Number of CUDA devices (0 without a GPU; never fails). */
int32_t pc_device_count(void);
/* Select the CUDA device used by handles created afterwards on this thread. */
pc_status pc_set_device(int32_t device);
/* Total number of kernels this library has launched in this process. */
uint64_t pc_launch_count(void);
/* Device memory freed by the library stays cached in each device's
 * stream-ordered pool for reuse by later handles; this returns it to the
 * device.  Call it with no handle in use. */
pc_status pc_release_cached_memory(void);
/* Page-lock (or release) a caller buffer so host<->device copies are DMA. */
pc_status pc_host_register(void* ptr, size_t bytes);
pc_status pc_host_unregister(void* ptr);
/* Self-test of the bounded grid barrier that the persistent kernels (k-core)
 * use: `rounds` barriers over a cooperative grid on `device`, checking that
 * no CTA passes a barrier early (*mismatches counts violations, 0 expected).
 * With absent_cta >= 0 that CTA never arrives: the other CTAs' waits run out
 * after limit_ms and the call returns PC_ERR_TIMEOUT with the device still
 * usable.  Not part of the reference interface; a diagnostic. */
pc_status pc_selftest_grid_barrier(int32_t device, int32_t rounds, int32_t absent_cta, uint32_t limit_ms,
                                   uint32_t* mismatches);

/* ---- graph (class Graph, src/Graph.hpp:38-103) ------------------------- */

#define PC_GRAPH_NO_VALIDATE 1u /* skip the device-side CSR checks */

/* Upload a symmetric CSR (rows strictly ascending, no self-loops, ids in
 * [0,n)).  weights may be NULL.  Replaces Graph::Graph(csrdir, is_weighted)
 * (src/Graph.cpp:92-137) and Graph::Graph(adj_list) (src/Graph.cpp:139-149):
 * the arrays are exactly the contents of csr_vlist.bin / csr_elist.bin /
 * csr_weight.bin.  Unless PC_GRAPH_NO_VALIDATE, the device checks that
 * offsets are monotone, ids in range, rows strictly ascending, no self-loops,
 * the adjacency symmetric (a two-way 64-bit fingerprint of the edge multiset)
 * and weights in [0, 2^30), and returns PC_ERR_INVALID_INPUT otherwise. */
pc_status pc_graph_create(const uint64_t* vlist, const int32_t* elist, const int32_t* weights,
                          uint64_t n, uint64_t m, uint32_t flags, pc_graph** out);
pc_status pc_graph_destroy(pc_graph* g);
/* Graph::get_vertex_num / get_edge_num / is_weighted (src/Graph.cpp:172-174, 288-294). */
pc_status pc_graph_info(const pc_graph* g, uint64_t* n, uint64_t* m, int32_t* weighted);
/* Opaque cudaStream_t of the handle (for event timing by the caller). */
void* pc_graph_stream(const pc_graph* g);

/* ---- ingest on the device ------------------------------------------------ */

#define PC_INGEST_DEGREE_RELABEL 1u /* relabel by descending degree, ties by id */

/* Build a graph on the device from a raw edge stream (host arrays, nedges
 * pairs, ids in [0, n)): both directions of every edge, self-loops dropped,
 * rows sorted and deduplicated -- the adjacency build of the text loader
 * Graph::Graph(file) (src/Graph.cpp:59-85, after parsing and without its id
 * shift) and of the preprocess tool (src/preprocess.cpp:5-45).  With
 * PC_INGEST_DEGREE_RELABEL the ids are relabelled by descending degree (ties
 * by ascending id) and old2new (n entries, may be NULL) receives the map.
 * Radix sort + unique + one pass on the device; the result equals the host
 * builder's arrays bit for bit. */
pc_status pc_graph_from_edges(const uint32_t* src, const uint32_t* dst, uint64_t nedges, uint64_t n, uint32_t flags,
                              int32_t* old2new, pc_graph** out);
/* Seeded synthetic graphs generated and built on the device; identical to
 * pc_synth_rmat / pc_synth_er below (same counter-based edge streams). */
pc_status pc_graph_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, uint32_t flags, pc_graph** out);
pc_status pc_graph_er(uint32_t scale, uint64_t nedges, uint64_t seed, uint32_t flags, pc_graph** out);
/* Symmetric integer weights in [1, wmax] keyed on the unordered endpoint
 * pair, computed on the device (= pc_synth_add_weights).  The preprocess
 * tool's weight file (src/preprocess.cpp:14-24) is the host path
 * (pc::Graph::add_reference_weights).  Fails while a partitioned view of g
 * exists. */
pc_status pc_graph_add_weights(pc_graph* g, uint64_t seed, int32_t wmax);
/* Copy the device CSR to host arrays (n+1 offsets, m ids, m weights; any may
 * be NULL): the contents of csr_vlist.bin / csr_elist.bin / csr_weight.bin
 * (Graph::save_as_csr_binfile, src/Graph.cpp:296-307). */
pc_status pc_graph_download(const pc_graph* g, uint64_t* vlist, int32_t* elist, int32_t* weights);

/* ---- partitioned graph (class Partitioned_Graph, src/Graph.hpp:105-155) -- */

/* Build the partitioned view.  Replaces Partitioned_Graph::Partitioned_Graph
 * (src/Graph.cpp:1017-1069).  v2p[u] in [0, P) for all u; P = max(v2p) + 1
 * as in the reference (src/Graph.cpp:1021).  v2p == NULL means one partition
 * (the unpartitioned Graph:: algorithms).  Vertex ids seen by the caller stay
 * the original ids until pc_pgraph_reorder() is called. */
pc_status pc_partition(pc_graph* g, const int32_t* v2p, pc_pgraph** out);
pc_status pc_pgraph_destroy(pc_pgraph* pg);
/* get_vertex_num / get_edge_num / get_partition_num (src/Graph.cpp:1210-1220). */
pc_status pc_pgraph_info(const pc_pgraph* pg, uint64_t* n, uint64_t* m, int32_t* partitions);
/* Partitioned_Graph::reorder (src/Graph.cpp:1665-1699): from now on vertex ids
 * in inputs and outputs are the partition-contiguous ids (partition by
 * partition, ascending original id inside a partition). */
pc_status pc_pgraph_reorder(pc_pgraph* pg);
/* Current id of original vertex u (identity before reorder). */
pc_status pc_pgraph_vertex_map(const pc_pgraph* pg, int32_t* old2new /* n */);
/* Materialise the reference's layout: vlist[k*n+u] .. vlist[k*n+u+1] is
 * N_k(u) inside elist, partition-major (src/Graph.cpp:1038-1067); weights
 * follow elist when the graph is weighted (may be NULL).  vlist has P*n+1
 * entries, elist/weights m.  Meant for small graphs and parity tests. */
pc_status pc_pgraph_layout(pc_pgraph* pg, uint64_t* vlist, int32_t* elist, int32_t* weights);
/* Graph::greedy_partition (src/Graph.cpp:898-967) on the GPU, seeded: the
 * vertices with degree >= P, in descending-degree order, spread their
 * unplaced neighbours over the partitions by the reference's quotas
 * max(0, deg/P - placed_i); all other vertices get a seeded random
 * partition (the reference's rule gives them zero quotas).  Heavy vertices
 * run in waves of 64; a vertex does not see what the others of its wave
 * place, the only difference from the sequential rule.  P <= 16384.
 * v2p receives n partition ids. */
pc_status pc_greedy_partition(pc_graph* g, int32_t P, uint64_t seed, int32_t* v2p);
/* evaluate_partition (src/Graph.cpp:1460-1473): max part degree, max degree. */
pc_status pc_pgraph_evaluate(pc_pgraph* pg, int64_t* max_part_deg, int64_t* max_deg, double* balance_ratio);

/* ---- intersection algorithms ------------------------------------------- */

/* Intersection methods of the reference. */
#define PC_METHOD_MERGE 0     /* *_merge: T (each triangle once)          */
#define PC_METHOD_GALLOPING 1 /* *_galloping: sum over ordered (u,v) = 6T */

/* Kernel variants (per-partition choices; see pc_tc_ex). */
#define PC_VARIANT_AUTO -1       /* learned selector if trained, else heuristic */
#define PC_VARIANT_HEURISTIC -2  /* plain autotuned heuristic                    */
#define PC_VARIANT_BITMAP_WARP 0 /* pivot bitmap in smem, warp per in-neighbour  */
#define PC_VARIANT_BITMAP_GROUP8 1 /* pivot bitmap, 8 lanes per in-neighbour     */
#define PC_VARIANT_BITMAP_LANE 2 /* pivot bitmap, one lane per in-neighbour      */
#define PC_VARIANT_HASH_WARP 3   /* warp-private pivot hash, lane per in-nbr     */
#define PC_VARIANT_MERGE_LANE 4  /* threshold merge, lane per edge (reference)   */
#define PC_VARIANT_GALLOP_LANE 5 /* binary search, lane per edge                 */
#define PC_VARIANT_MATRIX 6      /* hub units (ids < 2^16, contiguous partitions):
                                    pivot bitmap rows resident in L2, in-neighbour
                                    major, word-AND/popcount or bit probes       */
#define PC_NUM_VARIANTS 7

typedef struct {
    double kernel_ms;      /* device time of the intersection kernels (CUDA events) */
    uint64_t launches;     /* kernels launched by the call                          */
    uint64_t scan_bound;   /* sum over in-edges (c->b) of |N(c) & [0,c)|: bound on scanned ids */
    int32_t partitions;    /* number of partitions planned                          */
    int32_t variant_hist[PC_NUM_VARIANTS]; /* partitions per chosen variant         */
    int32_t selector;      /* 0 forced variant, 1 heuristic, 2 learned              */
} pc_tc_stats;

/* Partitioned_Graph::solve_triangle_counting_merge (src/Graph.cpp:1346-1362)
 * and ..._galloping (src/Graph.cpp:1326-1344); Graph::solve_triangle_counting_*
 * (src/Graph.cpp:342-368) on a one-partition view. */
pc_status pc_tc(pc_pgraph* pg, int32_t method, uint64_t* count);
pc_status pc_tc_ex(pc_pgraph* pg, int32_t method, int32_t variant, uint64_t* count, pc_tc_stats* stats);

/* Partitioned_Graph::solve_lcc_merge / _galloping (src/Graph.cpp:2197-2261);
 * Graph::solve_lcc_* (src/Graph.cpp:814-840).  out[n]: numerator / (d(d-1)),
 * d = 0 -> 0, d = 1 -> NaN, as the reference computes it. */
pc_status pc_lcc(pc_pgraph* pg, int32_t method, double* out);

/* All-edge Jaccard: out[e] for every CSR entry e = (u, v) in the order of the
 * graph's csr_elist: c / (d(u) + d(v) - c) with c = |N(u) & N(v)|, the
 * formula of Graph::solve_jsim_merge (src/Graph.cpp:798-812), rounded to fp32. */
pc_status pc_jaccard_edges(pc_pgraph* pg, float* out);
/* Graph::solve_jsim_merge over a query list (src/Graph.cpp:798-812):
 * out[i*nq+j] = J(q[i], q[j]) in fp64. */
pc_status pc_jaccard_queries(pc_pgraph* pg, const int32_t* queries, int32_t nq, double* out);

/* Partitioned_Graph::batch_cnt_common_neis_merge / _galloping over pairs
 * (src/Graph.cpp:1382-1393, 1421-1432): out[i] = |N(a_i) & N(b_i)|. */
pc_status pc_batch_count_pairs(pc_pgraph* pg, const int32_t* pairs /* 2*nq */, uint64_t nq, uint64_t* out);
/* ... over k-sets (src/Graph.cpp:1395-1406, 1434-1445): out[i] = |AND_j N(s_ij)|;
 * set i is ids[offsets[i] .. offsets[i+1]) (at least 2 vertices). */
pc_status pc_batch_count_sets(pc_pgraph* pg, const int32_t* ids, const uint64_t* offsets, uint64_t nq, uint64_t* out);

/* Friend triangles around root (Partitioned_Graph::solve_friend_triangle_merge
 * and _galloping, src/Graph.cpp:1222-1264; Graph:: forms src/Graph.cpp:309-340):
 * the sum over positions j < k of nodes, both not the root, of
 * |N(root) & N(nodes[j]) & N(nodes[k])|.  Both reference methods give this
 * number.  Computed without enumerating the pairs: for every w in N(root),
 * c_w positions are adjacent to it, and the sum is that of c_w (c_w - 1) / 2. */
pc_status pc_friend_triangle(pc_pgraph* pg, int32_t root, const int32_t* nodes, uint64_t nn, uint64_t* out);
/* Partitioned_Graph::solve_square_counting (src/Graph.cpp:1291-1324): the
 * sum over u and v, w in N(u) with w < v < u of |N(v) & N(w) & [0, w)|, in
 * the caller's vertex ids (after pc_pgraph_reorder, the reordered ones). */
pc_status pc_square_count(pc_pgraph* pg, uint64_t* out);

/* ---- frontier algorithms ----------------------------------------------- */

/* Partitioned_Graph::solve_bfs (src/Graph.cpp:1701-1762) output convention:
 * rank[src] = -1, rank[v] = BFS level (>= 1), unreached = INT32_MAX. */
pc_status pc_bfs(pc_pgraph* pg, int32_t src, int32_t* rank);
/* Partitioned_Graph::solve_sssp (src/Graph.cpp:2263-2309) / Graph::solve_sssp
 * (src/Graph.cpp:842-868): exact distances with the int32 weights,
 * unreached = INT32_MAX / 2.  Requires a weighted graph.  pc_sssp is
 * pc_sssp_ex(PC_SSSP_AUTO, delta 0). */
pc_status pc_sssp(pc_pgraph* pg, int32_t src, int32_t* dist);
/* The schedule of the relaxations, which never changes the result (both are
 * label-correcting and end at the exact distances):
 *   PC_SSSP_BELLMAN_FORD   frontier Bellman-Ford, the reference's partitioned
 *                          schedule (src/Graph.cpp:2263-2309): every improved
 *                          vertex is relaxed in the next round;
 *   PC_SSSP_DELTA_STEPPING delta-stepping (near/far piles): only vertices whose
 *                          distance is below the current bucket bound are
 *                          relaxed; buckets are `delta` wide (0: 8 x mean
 *                          weight, computed on the device);
 *   PC_SSSP_AUTO           delta-stepping with delta chosen from the graph. */
#define PC_SSSP_AUTO 0
#define PC_SSSP_BELLMAN_FORD 1
#define PC_SSSP_DELTA_STEPPING 2
pc_status pc_sssp_ex(pc_pgraph* pg, int32_t src, int32_t method, int32_t delta, int32_t* dist);
/* Partitioned_Graph::page_rank (src/Graph.cpp:1555-1602): x0 = d/(damping n),
 * x[v] <- (1-damping)/n + sum_{u in N(v)} x[u] * damping / d(u), in fp32.
 * init != NULL starts from the caller's vector instead, which is
 * Graph::page_rank (src/Graph.cpp:534-554; the same recurrence). */
pc_status pc_pagerank(pc_pgraph* pg, float damping, int32_t iterations, const float* init, float* out);
/* The same recurrence in fp64 (the FP64 form of the reference arithmetic). */
pc_status pc_pagerank_f64(pc_pgraph* pg, double damping, int32_t iterations, const double* init, double* out);
/* Partitioned_Graph::solve_kcore (src/Graph.cpp:1863-1942): core numbers. */
pc_status pc_kcore(pc_pgraph* pg, int32_t* core, int32_t* largest_core);
/* Partitioned_Graph::solve_mis (src/Graph.cpp:1944-2044) / Graph::solve_mis
 * (src/Graph.cpp:721-780): lexicographically-first maximal independent set
 * by vertex id; res[u] = 1 if u is in the set. */
pc_status pc_mis(pc_pgraph* pg, int32_t* res);
/* The same greedy rule with seed-hashed priorities: vertices ordered by
 * (hash(seed, id), id) instead of id -- the reference run on ids relabelled
 * by ascending hash, mapped back. */
pc_status pc_mis_hashed(pc_pgraph* pg, uint64_t seed, int32_t* res);
/* Partitioned_Graph::solve_cdlp (src/Graph.cpp:1843-1861): labels[u] <- max
 * label over N(u) (0 for isolated u), iterations times; in/out. */
pc_status pc_cdlp(pc_pgraph* pg, int32_t iterations, int32_t* labels);

/* ---- allocation-free entry point ------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory (their GPU memory belongs to another allocator or pool, or their
 * path must not risk an allocation's synchronisation or latency): the
 * triangle count -- each triangle once, as PC_METHOD_MERGE -- of a symmetric
 * CSR the caller already holds in device memory (d_vlist: n+1 uint64
 * offsets; d_elist: m int32 ids, rows strictly ascending, no self-loops).
 * Nothing is allocated: the temporaries live in a fixed array inside the
 * library image (about 4 MiB per GPU, held until the process exits), which
 * caps n at 2^20 vertices; larger graphs return PC_ERR_INVALID_INPUT.  The
 * CSR is checked only as far as memory safety needs (offsets non-decreasing
 * and ending at m, neighbour ids in [0, n)); a violation returns
 * PC_ERR_INVALID_INPUT.  Each call looks up that array's device address
 * (cudaGetSymbolAddress) in the current context.  Runs on the current
 * device, on `stream` (NULL: the legacy default stream), and is synchronous:
 * it returns once *count is written, so it must not be called while
 * `stream`, or any stream in global capture mode, is being captured.  Every
 * call shares the array, which keeps the previous call's contents (the
 * counters are cleared at the start of each call): calls that overlap on the
 * GPU race. */
pc_status pc_tc_count_noalloc(const uint64_t* d_vlist, const int32_t* d_elist, uint64_t n, uint64_t m,
                              void* stream, uint64_t* count);

/* ---- many graphs in one launch ---------------------------------------------
 * No counterpart in the reference (which runs one graph per call).  G
 * independent graphs packed in one CSR arena with arena-wide vertex ids:
 * graph g owns vertices [voff[g], voff[g+1]) and no edge joins two graphs.
 * pc_batch_run computes, for every graph, the tasks requested in one
 * persistent-kernel launch replayed from a captured CUDA graph:
 *   PC_BATCH_TC  tc[g]   triangles of graph g (solve_triangle_counting_merge);
 *   PC_BATCH_LCC lcc[v]  Graph::solve_lcc_merge per arena vertex;
 *   PC_BATCH_BFS bfs[v]  BFS level from graph g's first vertex, in
 *                        Partitioned_Graph::solve_bfs's convention. */
typedef struct pc_batch pc_batch;
#define PC_BATCH_TC 1u
#define PC_BATCH_LCC 2u
#define PC_BATCH_BFS 4u
typedef struct {
    double ms;           /* device time of the replayed launch (CUDA events) */
    uint32_t items;      /* (graph, task) work items */
    int32_t threads;     /* threads per CTA */
    int32_t ctas_per_sm; /* persistent CTAs per SM */
    int32_t order;       /* 0 largest graphs first, 1 graph order */
} pc_batch_stats;
pc_status pc_batch_create(const uint64_t* vlist, const int32_t* elist, uint64_t N, uint64_t M, const uint64_t* voff,
                          uint32_t G, pc_batch** out);
pc_status pc_batch_destroy(pc_batch* b);
pc_status pc_batch_run(pc_batch* b, uint32_t tasks, uint64_t* tc, double* lcc, int32_t* bfs, pc_batch_stats* stats);
/* Schedule: threads 256|512, ctas_per_sm 1..4, order 0|1. */
pc_status pc_batch_set_schedule(pc_batch* b, int32_t threads, int32_t ctas_per_sm, int32_t order);
/* Times every schedule candidate on this batch and keeps the fastest. */
pc_status pc_batch_autotune(pc_batch* b, uint32_t tasks, pc_batch_stats* best);

/* ---- per-partition kernel selection (no counterpart in the reference: the
 *      reference runs one scalar merge everywhere) ------------------------- */

/* Planning units: partitions, split into tiles of at most 16384 vertices. */
#define PC_SELECTOR_FEATURES 10 /* raw features per unit */
#define PC_MLP_IN 12
#define PC_MLP_HIDDEN 64
#define PC_MLP_OUT PC_NUM_VARIANTS
pc_status pc_tc_units(pc_pgraph* pg, int32_t* nunits);
/* Raw features per unit: pivots, in-edges, sum |N+(b)|, max |N+(b)|, max id+1,
 * sum of in-neighbour prefix lengths, mean and variance of log2(1+degree),
 * fraction of in-neighbours with a prefix >= 32, in-edges per pivot. */
pc_status pc_tc_unit_features(pc_pgraph* pg, float* feats /* nunits*PC_SELECTOR_FEATURES */, int32_t cap);
/* Variant chosen per unit (-1: no work) under a selection mode. */
pc_status pc_tc_plan(pc_pgraph* pg, int32_t variant, int8_t* assign, int32_t cap);
/* Device time of one variant on one unit alone, with its (partial) count. */
pc_status pc_tc_time_unit(pc_pgraph* pg, int32_t unit, int32_t variant, double* ms, uint64_t* count);
/* Training data: time every feasible variant on up to max_units units of pg
 * (heaviest first, then a stride over the rest), best of `repeats`; checks
 * that all variants return the same count. */
pc_status pc_selector_collect(pc_pgraph* pg, int32_t max_units, int32_t repeats, int32_t* samples_added);
/* Training data measured inside full runs: each variant runs on every unit it
 * can take in one profiled call (best of `repeats`); the kernels charge their
 * per-item warp-cycles to the units, and each unit's cost is its share of the
 * measured launch time.  One sample per unit with work; counts are checked
 * across the variants that ran on the same units. */
pc_status pc_selector_collect_insitu(pc_pgraph* pg, int32_t repeats, int32_t* samples_added);
int32_t pc_selector_num_samples(void);
pc_status pc_selector_get_samples(float* feats, float* log_ms, uint8_t* mask, int32_t cap);
pc_status pc_selector_add_samples(const float* feats, const float* log_ms, const uint8_t* mask, int32_t count);
/* Train the MLP on the GPU (full batch, Adam) on the collected samples. */
pc_status pc_selector_train(int32_t steps, float lr, uint64_t seed, float* final_loss);
/* The judge chosen at training: the learned choice replaces the heuristic's
 * only when predicted faster by more than exp(log_margin) (+inf: never), the
 * margin with the lowest measured total on held-out collection groups
 * (leave-one-group-out); heldout_gain = heuristic total / judged total there
 * (0 when fewer than two groups were collected). */
pc_status pc_selector_judge(double* log_margin, double* heldout_gain);
/* Predicted log(ms) per variant for raw unit features. */
pc_status pc_selector_predict(const float* feats, int32_t count, float* log_ms);
/* Grid-search the heuristic's thresholds on the collected samples. */
pc_status pc_selector_autotune(double* tuned /* 4 */);
/* Two-stage autotuning: the k best threshold sets by the same grid search on
 * the collected samples (distinct plans only), plus the thresholds in force,
 * are each applied and timed on the npg graph views (the heuristic plan's
 * counting time, median of `repeats` after one warm-up call).  Every view
 * weighs alike: the kept set has the lowest sum over views of its time over
 * the fastest set's time there; measured_ms is its summed time.  The views
 * should be graphs other than the ones the plan is measured on. */
pc_status pc_selector_autotune_measured(pc_pgraph* const* pgs, int32_t npg, int32_t k, int32_t repeats,
                                        double* tuned /* 4 */, double* measured_ms);
/* Heuristic thresholds: in-edges per pivot for a shared-memory or resident
 * bitmap form; mean prefix length for 32 lanes, for 8 lanes, and for the
 * matrix form (1e30 = never). */
pc_status pc_selector_get_heuristic(double* params /* 4 */);
pc_status pc_selector_set_heuristic(const double* params /* 4 */);
pc_status pc_selector_clear(void);
int32_t pc_selector_trained(void);
/* on == 0 makes PC_VARIANT_AUTO use the heuristic even when trained. */
pc_status pc_selector_enable(int32_t on);
pc_status pc_selector_save(const char* path);
pc_status pc_selector_load(const char* path);
/* The MLP's GPU kernels, exposed for gradient checks: parameters are
 * W1[H][IN] b1[H] W2[H][H] b2[H] W3[OUT][H] b3[OUT]; loss is the mean squared
 * error over masked outputs. */
int32_t pc_mlp_num_params(void);
pc_status pc_mlp_forward(const float* params, const float* x, int32_t batch, float* y);
pc_status pc_mlp_loss_grad(const float* params, const float* x, const float* y, const uint8_t* mask, int32_t batch,
                           float* loss, float* grad);
/* The same with each sample's squared errors weighted by weights[batch]
 * (NULL: all 1): the loss the selector's training minimises, with every
 * unit weighted by the measured time of its fastest variant. */
pc_status pc_mlp_loss_grad_weighted(const float* params, const float* x, const float* y, const uint8_t* mask,
                                    const float* weights, int32_t batch, float* loss, float* grad);
pc_status pc_mlp_train_steps(float* params, const float* x, const float* y, const uint8_t* mask, int32_t batch,
                             int32_t steps, float lr, float* final_loss);

/* ---- synthetic inputs (seeded; identical on host and device) ----------- */

typedef struct pc_host_csr pc_host_csr;
/* RMAT(0.57, 0.19, 0.19, 0.05), 2^scale vertices, edge_factor * 2^scale draws,
 * symmetrised, self-loops and duplicates dropped, rows sorted; relabel != 0
 * relabels by descending degree (ties by id). */
pc_status pc_synth_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, int32_t relabel, pc_host_csr** out);
/* Erdos-Renyi G(2^scale, nedges) draw, same post-processing. */
pc_status pc_synth_er(uint32_t scale, uint64_t nedges, uint64_t seed, int32_t relabel, pc_host_csr** out);
/* Chung-Lu expected-degree graph, exponent beta, expected max degree dmax. */
pc_status pc_synth_chung_lu(uint32_t scale, uint64_t nedges, double beta, uint64_t dmax, uint64_t seed,
                            int32_t relabel, pc_host_csr** out);
/* Symmetric integer weights in [1, wmax] keyed on the endpoint pair. */
pc_status pc_synth_add_weights(pc_host_csr* g, uint64_t seed, int32_t wmax);
/* Borrow the arrays (valid until pc_host_csr_free). weights NULL if none. */
pc_status pc_host_csr_arrays(const pc_host_csr* g, uint64_t* n, uint64_t* m, const uint64_t** vlist,
                             const int32_t** elist, const int32_t** weights);
/* Read / write the reference's binary CSR files <dir>/csr_{vlist,elist,weight}.bin
 * (Graph::Graph(csrdir, bool) src/Graph.cpp:92-137, save_as_csr_binfile src/Graph.cpp:595-605). */
pc_status pc_host_csr_load(const char* dir, int32_t weighted, pc_host_csr** out);
pc_status pc_host_csr_save(const pc_host_csr* g, const char* dir);
/* Wrap caller arrays (copied) into a host CSR. */
pc_status pc_host_csr_from_arrays(const uint64_t* vlist, const int32_t* elist, const int32_t* weights,
                                  uint64_t n, uint64_t m, pc_host_csr** out);
pc_status pc_host_csr_free(pc_host_csr* g);
/* G seeded RMAT graphs in one arena: graph g has scale in [smin, smax] and
 * edge factor in [emin, emax] drawn from (seed, g), RMAT seed g, and is
 * symmetrised, deduplicated and degree-relabelled; voff (G+1) receives the
 * arena offsets of the graphs. */
pc_status pc_synth_rmat_batch(uint32_t G, uint32_t smin, uint32_t smax, uint32_t emin, uint32_t emax, uint64_t seed,
                              pc_host_csr** out, uint64_t* voff);
/* The sequential seeded greedy partitioner on the host (src/Graph.cpp:898-967
 * with one std::mt19937 in place of random_device and rand()). */
pc_status pc_host_greedy_partition(const uint64_t* vlist, const int32_t* elist, uint64_t n, int32_t P, uint64_t seed,
                                   int32_t* v2p);
/* The priorities pc_mis_hashed orders vertices by: out[v] for v < n. */
pc_status pc_synth_vertex_priority(uint64_t seed, uint64_t n, uint64_t* out);

#ifdef __cplusplus
}
#endif
#endif /* PC_H */
