"""GPU parity: every algorithm of libpc.so (through its C ABI) against the CPU
oracle and the reference's own golden outputs.

Bars: integer results bit-exact; LCC / Jaccard bit-exact too (the integer
numerators are exact and the division is one IEEE operation, as in the
reference); PageRank fp64 within 1e-6 relative of the FP64 oracle (observed
~1e-15); PageRank fp32 (fp32 vectors, fp64 row sums) within 1e-6 relative of
the FP64 oracle too; against the reference's own fp32 run, whose fp32 row sums
over up to 10^4 terms drift from FP64, within 1e-4."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN_GRAPHS, INT_MAX, golden_summary, load_golden, small_graphs

pytestmark = pytest.mark.gpu

PR_F64_RTOL = 1e-6
PR_F32_RTOL = 1e-6      # fp32 output against the FP64 oracle
PR_F32_REF_RTOL = 1e-4  # fp32 output against the reference's fp32 output


def partitions(n, rng):
    out = {"P1": None}
    if n >= 3:
        out["P3"] = (np.arange(n) * 3 // n).astype(np.int32)
    if n >= 1:
        out["P64"] = (np.arange(n) * min(64, n) // n).astype(np.int32)
        out["Pn"] = np.arange(n, dtype=np.int32)
        out["rand7"] = rng.integers(0, 7, n).astype(np.int32)
    return out


def relabel_csr(vl, el, old2new):
    """CSR of the graph with ids mapped by old2new (rows re-sorted)."""
    n = vl.size - 1
    new2old = np.empty(n, np.int64)
    new2old[old2new] = np.arange(n)
    deg = np.diff(vl).astype(np.int64)
    nvl = np.zeros(n + 1, np.uint64)
    np.cumsum(deg[new2old], out=nvl[1:])
    nel = np.empty_like(el)
    for r in range(n):
        o = new2old[r]
        row = np.sort(old2new[el[vl[o]:vl[o + 1]]])
        nel[nvl[r]:nvl[r + 1]] = row
    return nvl, nel


@pytest.fixture(scope="module")
def cases(gpu):
    pc = gpu
    rng = np.random.default_rng(2024)
    out = []
    for name, vl, el, w in small_graphs(pc):
        if w is None:
            w = np.ones(el.size, np.int32)
        g = pc.Graph(vlist=vl, elist=el, weights=w)
        for pname, v2p in partitions(vl.size - 1, rng).items():
            out.append((f"{name}-{pname}", vl, el, w, v2p, g))
    return out


def _pg(pc, g, v2p):
    return pc.Partitioned_Graph(g, v2p)


def test_triangle_count_all_variants(gpu, O, cases):
    pc = gpu
    for cid, vl, el, w, v2p, g in cases:
        t = O.tc_merge(vl, el)
        pg = _pg(pc, g, v2p)
        contiguous = v2p is None or bool(np.all(np.diff(v2p) >= 0))
        f = pc.selector.unit_features(pg)
        work = (f[:, 1] > 0) & (f[:, 2] > 0)
        # (a graph without edges runs no kernel, so nothing is refused)
        matrix_ok = (contiguous and not bool(np.any(work & (f[:, 4] > 1 << 16)))) or el.size == 0
        for vname, v in list(pc.VARIANTS.items()) + [("heuristic", pc.VARIANT_HEURISTIC), ("auto", pc.VARIANT_AUTO)]:
            if vname == "matrix" and not matrix_ok:
                with pytest.raises(pc.PCError):  # needs units that are id ranges below 2^16
                    pg.triangle_count(variant=v)
                continue
            got = pg.triangle_count(variant=v)
            assert got == t, (cid, vname, got, t)
        assert pg.solve_triangle_counting_galloping() == 6 * t, cid
        pg.close()
    for name, vl, el, w in small_graphs(pc)[:4]:
        assert pc.Graph(vlist=vl, elist=el).solve_triangle_counting_merge() == O.tc_merge(vl, el)


def test_layout_matches_reference_construction(gpu, O, cases):
    pc = gpu
    for cid, vl, el, w, v2p, g in cases:
        n = vl.size - 1
        if v2p is None or n * (int(v2p.max()) + 1 if n else 1) > 4_000_000:
            continue
        pg = _pg(pc, g, v2p)
        lv, le, lw = pg.layout()
        ov, oe, ow = O.layout(vl, el, w, v2p)
        np.testing.assert_array_equal(lv, ov, err_msg=cid)
        np.testing.assert_array_equal(le, oe, err_msg=cid)
        np.testing.assert_array_equal(lw, ow, err_msg=cid)
        pg.close()


def test_layout_after_reorder(gpu, O, cases):
    """Partitioned_Graph::reorder: new ids partition by partition (ascending
    old id inside), rows and neighbour ids in the new ids."""
    pc = gpu
    for cid, vl, el, w, v2p, g in cases:
        if v2p is None or not cid.endswith("rand7"):
            continue
        n = vl.size - 1
        order = np.lexsort((np.arange(n), v2p))  # new -> old
        old2new = np.empty(n, np.int32)
        old2new[order] = np.arange(n, dtype=np.int32)
        pg = _pg(pc, g, v2p)
        pg.reorder()
        np.testing.assert_array_equal(pg.vertex_map(), old2new)
        lv, le, _ = pg.layout()
        P = int(v2p.max()) + 1
        # expected: for partition k, for new row r (old u = order[r]), N_k(u) mapped
        exp_v = np.zeros(P * n + 1, np.uint64)
        exp_e = []
        pos = 0
        for k in range(P):
            for r in range(n):
                u = order[r]
                exp_v[k * n + r] = pos
                row = el[vl[u]:vl[u + 1]]
                sub = row[v2p[row] == k]
                exp_e.extend(old2new[sub].tolist())
                pos += sub.size
        exp_v[P * n] = pos
        np.testing.assert_array_equal(lv, exp_v, err_msg=cid)
        np.testing.assert_array_equal(le, np.asarray(exp_e, np.int32), err_msg=cid)
        pg.close()


def test_lcc_and_jaccard(gpu, O, cases):
    pc = gpu
    for cid, vl, el, w, v2p, g in cases:
        pg = _pg(pc, g, v2p)
        ref = O.lcc(vl, el)
        for got in (pg.solve_lcc_merge(), pg.solve_lcc_galloping()):
            np.testing.assert_array_equal(np.isnan(got), np.isnan(ref), err_msg=cid)
            np.testing.assert_array_equal(got, ref, err_msg=cid)
        if el.size:
            exp = O.jaccard_edges(vl, el)
            np.testing.assert_array_equal(pg.jaccard_edges(), exp, err_msg=cid)
            # caller-owned output (pinned host memory, as a pinned torch tensor gives)
            import torch
            pinned = torch.full((el.size,), -1.0, dtype=torch.float32, pin_memory=True).numpy()
            assert pg.jaccard_edges(out=pinned) is pinned
            np.testing.assert_array_equal(pinned, exp, err_msg=cid)
            with pytest.raises(ValueError):
                pg.jaccard_edges(out=np.empty(el.size + 1, np.float32))
        n = vl.size - 1
        if n:
            q = np.unique(np.random.default_rng(3).integers(0, n, min(n, 20))).astype(np.int32)
            np.testing.assert_array_equal(pg.jaccard_queries(q), O.jaccard_queries(vl, el, q), err_msg=cid)
        pg.close()


def test_batch_counts(gpu, O, cases):
    pc = gpu
    rng = np.random.default_rng(5)
    for cid, vl, el, w, v2p, g in cases:
        n = vl.size - 1
        if n < 2:
            continue
        pg = _pg(pc, g, v2p)
        pairs = rng.integers(0, n, size=(200, 2)).astype(np.int32)
        np.testing.assert_array_equal(pg.batch_cnt_common_neis_merge(pairs), O.batch_pairs(vl, el, pairs), err_msg=cid)
        sets = [rng.integers(0, n, size=int(k)).astype(np.int32) for k in rng.integers(2, 6, size=50)]
        np.testing.assert_array_equal(pg.batch_cnt_common_neis_merge(sets), O.batch_sets(vl, el, sets), err_msg=cid)
        pg.close()


def test_frontier_algorithms(gpu, O, cases):
    pc = gpu
    for cid, vl, el, w, v2p, g in cases:
        n = vl.size - 1
        if n == 0:
            continue
        pg = _pg(pc, g, v2p)
        for src in {0, n // 2, n - 1}:
            np.testing.assert_array_equal(pg.solve_bfs(src), O.bfs(vl, el, src), err_msg=f"{cid} bfs {src}")
            want = O.sssp(vl, el, w, src)
            np.testing.assert_array_equal(pg.solve_sssp(src), want, err_msg=f"{cid} sssp {src}")
            # every schedule and bucket width ends at the same exact distances
            for method, delta in ((pc.SSSP_BELLMAN_FORD, 0), (pc.SSSP_DELTA_STEPPING, 0), (pc.SSSP_DELTA_STEPPING, 1),
                                  (pc.SSSP_DELTA_STEPPING, 37), (pc.SSSP_DELTA_STEPPING, 1 << 29)):
                np.testing.assert_array_equal(pg.solve_sssp(src, method=method, delta=delta), want,
                                              err_msg=f"{cid} sssp {src} method {method} delta {delta}")
        ref64 = O.pagerank_f64(vl, el, 0.85, 20)
        np.testing.assert_allclose(pg.page_rank(0.85, 20, fp64=True), ref64, rtol=PR_F64_RTOL, atol=0, err_msg=cid)
        np.testing.assert_allclose(pg.page_rank(0.85, 20).astype(np.float64), ref64, rtol=PR_F32_RTOL, atol=0,
                                   err_msg=cid)
        ones = np.ones(n)
        np.testing.assert_allclose(pg.page_rank(0.85, 5, init=ones, fp64=True),
                                   O.pagerank_f64(vl, el, 0.85, 5, init=ones), rtol=PR_F64_RTOL, atol=0)
        core, _ = O.kcore(vl, el)
        np.testing.assert_array_equal(pg.solve_kcore(), core, err_msg=cid)
        np.testing.assert_array_equal(pg.solve_mis(), O.mis(vl, el), err_msg=cid)
        prio = pc.vertex_priority(17, n)
        np.testing.assert_array_equal(pg.solve_mis(seed=17), O.mis(vl, el, priority=prio), err_msg=cid)
        lab = np.arange(n, dtype=np.int32)
        np.testing.assert_array_equal(pg.solve_cdlp(lab, 10), O.cdlp(vl, el, lab, 10), err_msg=cid)
        lab2 = np.random.default_rng(1).integers(0, 1000, n).astype(np.int32)
        np.testing.assert_array_equal(pg.solve_cdlp(lab2, 3), O.cdlp(vl, el, lab2, 3), err_msg=cid)
        pg.close()


def test_reordered_view_maps_ids(gpu, O, cases):
    """After reorder(), inputs and outputs use the new ids: results equal the
    oracle on the relabelled graph."""
    pc = gpu
    for cid, vl, el, w, v2p, g in cases:
        if v2p is None or not cid.endswith("rand7") or vl.size - 1 < 2:
            continue
        n = vl.size - 1
        pg = _pg(pc, g, v2p)
        pg.reorder()
        o2n = pg.vertex_map()
        nvl, nel = relabel_csr(vl, el, o2n)
        src = int(o2n[0])
        np.testing.assert_array_equal(pg.solve_bfs(src), O.bfs(nvl, nel, src), err_msg=cid)
        np.testing.assert_array_equal(pg.solve_mis(), O.mis(nvl, nel), err_msg=cid)
        np.testing.assert_array_equal(pg.solve_kcore(), O.kcore(nvl, nel)[0], err_msg=cid)
        ref = O.lcc(nvl, nel)
        np.testing.assert_array_equal(pg.solve_lcc_merge(), ref, err_msg=cid)
        lab = np.arange(n, dtype=np.int32)
        np.testing.assert_array_equal(pg.solve_cdlp(lab, 4), O.cdlp(nvl, nel, lab, 4), err_msg=cid)
        np.testing.assert_allclose(pg.page_rank(0.85, 10, fp64=True), O.pagerank_f64(nvl, nel, 0.85, 10),
                                   rtol=PR_F64_RTOL, atol=0)
        pairs = np.array([[0, 1], [1, n - 1]], np.int32)
        np.testing.assert_array_equal(pg.batch_cnt_common_neis_merge(pairs), O.batch_pairs(nvl, nel, pairs))
        pg.close()


@pytest.mark.parametrize("name", GOLDEN_GRAPHS)
def test_against_reference_golden(gpu, name):
    """GPU results equal the reference's own outputs (tests/golden/)."""
    pc = gpu
    d = load_golden(name)
    vl, el, w = d["vlist"], d["elist"], d["weights"]
    n = vl.size - 1
    g = pc.Graph(vlist=vl, elist=el, weights=w)
    pg = pc.Partitioned_Graph(g, d["v2p"])
    assert pg.solve_triangle_counting_merge() == int(d["tc_merge_partitioned"])
    assert pg.solve_triangle_counting_galloping() == int(d["tc_galloping_partitioned"])
    lv, le, _ = pg.layout()
    np.testing.assert_array_equal(lv, d["layout_vlist"])
    np.testing.assert_array_equal(le, d["layout_elist"])
    np.testing.assert_array_equal(pg.solve_lcc_merge(), d["lcc_partitioned"])
    if d["jsim_queries"].size:
        np.testing.assert_array_equal(pg.jaccard_queries(d["jsim_queries"]), d["jsim"])
    if "pairs" in d:
        np.testing.assert_array_equal(pg.batch_cnt_common_neis_merge(d["pairs"]), d["pair_counts_partitioned"])
        offs = d["set_offsets"].astype(np.int64)
        sets = [d["set_ids"][offs[i]:offs[i + 1]] for i in range(offs.size - 1)]
        np.testing.assert_array_equal(pg.batch_cnt_common_neis_merge(sets), d["set_counts_partitioned"])
    if n:
        np.testing.assert_array_equal(pg.solve_bfs(0), d["bfs_levels"])
        np.testing.assert_array_equal(pg.solve_sssp(0), d["sssp_partitioned"])
        np.testing.assert_array_equal(pg.solve_kcore(), d["kcore_partitioned"])
        np.testing.assert_array_equal(pg.solve_mis(), d["mis"])
        np.testing.assert_array_equal(pg.solve_cdlp(np.arange(n, dtype=np.int32), 10), d["cdlp_partitioned"])
        np.testing.assert_allclose(pg.page_rank(0.85, 20).astype(np.float64),
                                   d["pagerank_f32_partitioned"].astype(np.float64), rtol=PR_F32_REF_RTOL, atol=0)


def test_config1_rmat16(gpu, O):
    """RMAT scale 16, ef 16, seed 1, 64 equal-vertex partitions: TC, BFS from 0
    and PageRank (0.85, 20 iterations, fp64) against the oracle and the
    reference's recorded scalars."""
    pc = gpu
    s = golden_summary()
    h = pc.HostCSR.rmat(16, 16, 1).add_weights(seed=1, wmax=255)
    vl, el, w = h.arrays()
    n = vl.size - 1
    g = pc.Graph(vlist=vl, elist=el, weights=w)
    pg = pc.Partitioned_Graph(g, pc.equal_vertex_partition(n, 64))
    assert pg.get_partition_num() == 64
    assert pg.solve_triangle_counting_merge() == s["tc_merge_partitioned"]
    assert pg.solve_triangle_counting_galloping() == s["tc_galloping"]
    lev = pg.solve_bfs(0)
    np.testing.assert_array_equal(lev, O.bfs(vl, el, 0))
    assert int(lev[lev < INT_MAX].astype(np.int64).sum()) == s["bfs_levels_sum"]
    pr = pg.page_rank(0.85, 20, fp64=True)
    ref = O.pagerank_f64(vl, el, 0.85, 20)
    assert np.max(np.abs(pr - ref) / ref) <= PR_F64_RTOL
    core = pg.solve_kcore()
    assert int(core.astype(np.int64).sum()) == s["kcore_sum"]
    mis = pg.solve_mis()
    assert int(mis.sum()) == s["mis_size"]
    d = pg.solve_sssp(0)
    assert int(d[d < 2**31 // 2].astype(np.int64).sum()) == s["sssp_sum"]
    lab = pg.solve_cdlp(np.arange(n, dtype=np.int32), 10)
    assert int(lab.astype(np.int64).sum()) == s["cdlp_sum"]
    lcc = pg.solve_lcc_merge()
    assert int(np.isnan(lcc).sum()) == s["lcc_nan"]


@pytest.mark.parametrize("scale,P", [(16, 8), (19, 16)])
def test_matrix_form_on_hub_units(gpu, O, scale, P):
    """The in-neighbour-major form (resident pivot bitmap rows, word-AND and
    bit probes) on every unit whose ids are below 2^16 and whose rows fit
    100 MB, the other units by the usual kernels: exact counts, forced where
    every unit qualifies."""
    pc = gpu
    sel = pc.selector
    vl, el, _ = pc.HostCSR.rmat(scale, 16, 3).arrays()
    n = vl.size - 1
    t = O.tc_merge(vl, el)
    g = pc.Graph(vlist=vl, elist=el)
    pg = pc.Partitioned_Graph(g, pc.equal_vertex_partition(n, P))
    saved = sel.get_heuristic()
    try:
        sel.set_heuristic([1.0, 48.0, 6.0, 0.0])  # matrix wherever it is feasible
        c, st = pg.triangle_count(variant=pc.VARIANT_HEURISTIC, stats=True)
        assert c == t and st.variant_hist[pc.VARIANTS["matrix"]] > 0
        # LCC under the same plan (matrix units run the 32-lane bitmap kernel in
        # per-vertex mode), bit-exact with NaN at degree 1
        lcc = pg.solve_lcc_merge()
        want = O.lcc(vl, el)
        np.testing.assert_array_equal(np.isnan(lcc), np.isnan(want))
        np.testing.assert_array_equal(lcc, want)
        if n <= 1 << 16:
            assert pg.triangle_count(variant=pc.VARIANTS["matrix"]) == t
        else:
            with pytest.raises(pc.PCError):
                pg.triangle_count(variant=pc.VARIANTS["matrix"])
    finally:
        sel.set_heuristic(saved)
    pg.close()
    # non-contiguous partitions: the heuristic never picks the matrix form
    pg = pc.Partitioned_Graph(g, np.random.default_rng(1).integers(0, P, n).astype(np.int32))
    sel.set_heuristic([1.0, 48.0, 6.0, 0.0])
    try:
        c, st = pg.triangle_count(variant=pc.VARIANT_HEURISTIC, stats=True)
        assert c == t and st.variant_hist[pc.VARIANTS["matrix"]] == 0
    finally:
        sel.set_heuristic(saved)
    pg.close()
    g.close()


def test_bitmap_kernels_every_set_shape(gpu, O):
    """Forced bitmap variants on RMAT-20 with 64 partitions: units with pivot
    ids past 2^16 hold split sets (K = 2 in the count mode, K = 4 in the
    per-vertex mode of LCC).  Counts and LCC must equal the oracle's.  The
    per-edge mode's plain bitmaps of every size are covered by
    test_per_edge_mode_every_set_shape."""
    pc = gpu
    h = pc.HostCSR.rmat(20, 16, 5)
    vl, el, _ = h.arrays()
    n = vl.size - 1
    t = O.tc_merge(vl, el)
    pg = pc.Partitioned_Graph(pc.Graph(vlist=vl, elist=el), pc.equal_vertex_partition(n, 64))
    for name in ("bitmap_warp", "bitmap_group8", "bitmap_lane"):
        assert pg.triangle_count(variant=pc.VARIANTS[name]) == t, name
    assert pg.triangle_count(variant=pc.VARIANT_HEURISTIC) == t
    f = pc.selector.unit_features(pg)
    assert f[:, 1].sum() == el.size // 2  # every in-edge belongs to one unit
    assert (f[:, 0].sum(), f[:, 4].max()) == (n, n)
    # per-vertex mode (LCC) under a plan with the 8-lane bitmap kernel wherever
    # it is feasible: plain bitmaps below id 2^16, split sets above
    saved = pc.selector.get_heuristic()
    try:
        pc.selector.set_heuristic([0.0, 1e9, 0.0, 1e9])
        lcc = pg.solve_lcc_merge()
    finally:
        pc.selector.set_heuristic(saved)
    want = O.lcc(vl, el)
    np.testing.assert_array_equal(np.isnan(lcc), np.isnan(want))
    np.testing.assert_array_equal(lcc, want)


def _split_overflow_graph():
    """Pivot ids past 2^16, where the count mode's bitmap kernels hold a pivot
    set as a bitmap of the ids below 2^16 plus a 512-slot hash of the rest:
    pivot b1 has 600 neighbours in [2^16, b1) (more than the hash takes, so
    its high ids are found by binary search), pivot b2 has 100 (hashed); both
    have 50 in-neighbours c > b whose rows hit random low and high ids of the
    pivot's set."""
    rng = np.random.default_rng(77)
    L = 1 << 16
    high = np.arange(L, L + 600)
    low = np.arange(0, 100)
    b1, b2 = L + 700, L + 760
    edges = [(b1, int(x)) for x in high] + [(b1, int(x)) for x in low]
    edges += [(b2, int(x)) for x in high[:100]] + [(b2, int(x)) for x in low[:40]]
    for c in range(L + 800, L + 850):
        edges.append((c, b1))
        edges += [(c, int(x)) for x in rng.choice(np.concatenate([low, high]), 200, replace=False)]
    for c in range(L + 900, L + 950):
        edges.append((c, b2))
        edges += [(c, int(x)) for x in rng.choice(np.concatenate([low[:60], high[:150]]), 60, replace=False)]
    # some triangles among the high ids themselves
    for i in range(0, 590, 7):
        edges.append((int(high[i]), int(high[i + 3])))
        edges.append((int(high[i]), int(low[i % 100])))
        edges.append((int(high[i + 3]), int(low[i % 100])))
    from conftest import csr_from_edges
    return csr_from_edges(L + 1000, edges)


def test_split_pivot_sets(gpu, O):
    """Forced bitmap variants where pivot ids exceed 2^16: RMAT-18 with 16
    partitions, and a graph whose pivot sets overflow the split set's hash;
    the counts equal the oracle's."""
    pc = gpu
    cases = []
    vl, el, _ = pc.HostCSR.rmat(18, 16, 4).arrays()
    cases.append(("rmat18", vl, el, pc.equal_vertex_partition(vl.size - 1, 16)))
    vl, el = _split_overflow_graph()
    cases.append(("overflow-P1", vl, el, None))
    cases.append(("overflow-P5", vl, el, pc.equal_vertex_partition(vl.size - 1, 5)))
    for cid, vl, el, v2p in cases:
        t = O.tc_merge(vl, el)
        assert t > 0, cid
        pg = pc.Partitioned_Graph(pc.Graph(vlist=vl, elist=el), v2p)
        f = pc.selector.unit_features(pg)
        assert f[:, 4].max() > 1 << 16, cid
        for name in ("bitmap_warp", "bitmap_group8", "bitmap_lane"):
            assert pg.triangle_count(variant=pc.VARIANTS[name]) == t, (cid, name)
        assert pg.triangle_count(variant=pc.VARIANT_HEURISTIC) == t, cid
        assert pg.triangle_count() == t, cid
        # per-vertex mode (LCC) with split sets, under a bitmap plan
        saved = pc.selector.get_heuristic()
        try:
            pc.selector.set_heuristic([0.0, 1e9, 0.0, 1e9])
            lcc = pg.solve_lcc_merge()
        finally:
            pc.selector.set_heuristic(saved)
        want = O.lcc(vl, el)
        np.testing.assert_array_equal(np.isnan(lcc), np.isnan(want), err_msg=cid)
        np.testing.assert_array_equal(lcc, want, err_msg=cid)
        pg.close()


def test_per_edge_mode_every_set_shape(gpu, O):
    """All-edge Jaccard (per-edge mode, which keeps plain bitmaps for the ranks
    of its hits) under a plan with the 8-lane bitmap kernel wherever it is
    feasible, on a Chung-Lu graph with 2^20 vertices (exponent 2.1, 2^22
    edges, 4.9 M triangles) and 16 partitions: pivot ids up to 2^20 make the
    kernels share one bitmap among K = 1, 2, 4, 8 and 16 warps; LCC under the
    same plan uses split sets past 2^16.  Both equal the oracle's."""
    pc = gpu
    vl, el, _ = pc.HostCSR.chung_lu(20, 1 << 22, 2.1, 1 << 12, 3).arrays()
    n = vl.size - 1
    pg = pc.Partitioned_Graph(pc.Graph(vlist=vl, elist=el), pc.equal_vertex_partition(n, 16))
    assert pc.selector.unit_features(pg)[:, 4].max() > 1 << 19
    saved = pc.selector.get_heuristic()
    try:
        pc.selector.set_heuristic([0.0, 1e9, 0.0, 1e9])
        jac = pg.jaccard_edges()
        lcc = pg.solve_lcc_merge()
        c, st = pg.triangle_count(variant=pc.VARIANT_HEURISTIC, stats=True)
    finally:
        pc.selector.set_heuristic(saved)
    assert st.variant_hist[pc.VARIANTS["bitmap_group8"]] > 0
    assert c == O.tc_merge(vl, el)
    np.testing.assert_array_equal(jac, O.jaccard_edges(vl, el))
    want = O.lcc(vl, el)
    np.testing.assert_array_equal(np.isnan(lcc), np.isnan(want))
    np.testing.assert_array_equal(lcc, want)
    pg.close()
