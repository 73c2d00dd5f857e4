"""Generates the golden fixtures in tests/golden/ by running the REFERENCE itself.

The reference (PartitionAndConquer's src/Graph.cpp, unmodified) is compiled by
oracle/Makefile into oracle/_ref/libpcref.so; this script loads it through
oracle/oracle.py, runs its own member functions on small seeded graphs and
saves their outputs.  The CPU test suite then checks the C restatement
(oracle/pc_oracle.c) against these files, and the GPU suite checks libpc.so
against both.  Run from the repository root:

    python tests/golden/make_golden.py

The reference has no tests or fixtures of its own, so these outputs of the
reference's code are the pins.  The partitioned BFS of the reference does not
terminate (src/Graph.cpp:1717-1731 scans partition 0 only), so BFS levels come
from Graph::solve_bfs's parent tree (depth of each vertex).
"""
from __future__ import annotations

import json
import zlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import partitionandconquer_b200 as pc  # noqa: E402  (host generators only; no GPU needed)
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent


def csr_from_edges(n, edges):
    adj = [set() for _ in range(n)]
    for u, v in edges:
        if u != v:
            adj[u].add(v)
            adj[v].add(u)
    vl = np.zeros(n + 1, np.uint64)
    el = []
    for u in range(n):
        row = sorted(adj[u])
        el.extend(row)
        vl[u + 1] = vl[u] + len(row)
    return vl, np.asarray(el, np.int32)


def levels_from_parents(parents, src):
    """Depth of every vertex in Graph::solve_bfs's tree, in the partitioned
    output convention: src -1, depth r >= 1, unreached INT_MAX."""
    n = parents.size
    INF = 2**31 - 1
    lev = np.full(n, -2, np.int64)
    lev[src] = 0
    for v in range(n):
        if parents[v] == INF and v != src:
            lev[v] = -3
    def depth(v):
        path = []
        while lev[v] == -2:
            path.append(v)
            v = parents[v]
        d = lev[v]
        for x in reversed(path):
            d += 1
            lev[x] = d
        return d
    for v in range(n):
        if lev[v] == -2:
            depth(v)
    out = np.where(lev == -3, INF, lev).astype(np.int64)
    out[src] = -1
    return out.astype(np.int32)


def graphs():
    tiny_edges = [(0, 1), (1, 2), (2, 0), (2, 3), (3, 4), (4, 2), (0, 3)]
    yield "tiny", (*csr_from_edges(5, tiny_edges), None), 2
    yield "k6", (*csr_from_edges(6, [(i, j) for i in range(6) for j in range(i + 1, 6)]), None), 3
    yield "star", (*csr_from_edges(8, [(0, i) for i in range(1, 8)]), None), 2
    yield "path", (*csr_from_edges(8, [(i, i + 1) for i in range(7)]), None), 4
    yield "isolated", (np.zeros(6, np.uint64), np.zeros(0, np.int32), None), 2
    h = pc.HostCSR.rmat(10, 16, 3).add_weights(seed=3, wmax=255)
    yield "rmat10", h.arrays(), 8
    h = pc.HostCSR.er(10, 8192, 5).add_weights(seed=5, wmax=255)
    yield "er10", h.arrays(), 16


def run_reference(name, vl, el, w, P):
    n = vl.size - 1
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    v2p = pc.equal_vertex_partition(n, P)
    if w is None:
        w = np.ones(el.size, np.int32) if el.size else np.zeros(0, np.int32)
    R = O.Reference(vl, el, w=w, v2p=v2p, threads=4)
    # Partitioned paths that write shared state without atomics (SSSP's dist[]
    # and bitset, src/Graph.cpp:2286-2288; k-core's degrees[], :1930) lose
    # updates when several threads run them; they are pinned single-threaded.
    R1 = O.Reference(vl, el, w=w, v2p=v2p, threads=1)
    d = {"vlist": vl, "elist": el, "weights": w, "v2p": v2p}
    d["tc_merge"] = np.uint64(R.tc())
    d["tc_merge_partitioned"] = np.uint64(R.tc(partitioned=True))
    d["tc_galloping"] = np.uint64(R.tc(galloping=True))
    d["tc_galloping_partitioned"] = np.uint64(R.tc(partitioned=True, galloping=True))
    lv, le = R.layout()
    d["layout_vlist"], d["layout_elist"] = lv, le
    d["lcc"] = R.lcc()
    d["lcc_partitioned"] = R.lcc(partitioned=True)
    q = np.arange(min(n, 12), dtype=np.int32)
    d["jsim_queries"] = q
    d["jsim"] = R.jsim(q) if q.size else np.zeros(0)
    if n >= 2:
        pairs = rng.integers(0, n, size=(32, 2), dtype=np.int32)
        d["pairs"] = pairs
        d["pair_counts"] = R.batch_pairs(pairs)
        d["pair_counts_partitioned"] = R.batch_pairs(pairs, partitioned=True)
        sets = [rng.integers(0, n, size=int(k)).astype(np.int32) for k in rng.integers(2, 5, size=12)]
        d["set_ids"] = np.concatenate(sets)
        d["set_offsets"] = np.concatenate([[0], np.cumsum([len(s) for s in sets])]).astype(np.uint64)
        d["set_counts"] = R.batch_sets(sets)
        d["set_counts_partitioned"] = R.batch_sets(sets, partitioned=True)
        # friend triangles around the highest-degree vertex (root and a repeat inside the list)
        root = int(np.argmax(np.diff(vl.astype(np.int64))))
        nodes = rng.integers(0, n, size=24).astype(np.int32)
        nodes[3] = root
        nodes[5] = nodes[4]
        d["friend_root"] = np.int32(root)
        d["friend_nodes"] = nodes
        d["friend_merge"] = np.uint64(R.friend_triangle(root, nodes))
        d["friend_galloping"] = np.uint64(R.friend_triangle(root, nodes, galloping=True))
        d["friend_partitioned"] = np.uint64(R.friend_triangle(root, nodes, partitioned=True))
        d["friend_partitioned_galloping"] = np.uint64(R.friend_triangle(root, nodes, partitioned=True,
                                                                        galloping=True))
        d["squares_partitioned"] = np.uint64(R.square_count())
    if n:
        d["bfs_levels"] = levels_from_parents(R.bfs_parents(0), 0)
        d["sssp"] = R.sssp(0)
        d["sssp_partitioned"] = R1.sssp(0, partitioned=True)
        d["pagerank_f32_partitioned"] = R.pagerank(0.85, 20, partitioned=True)
        d["kcore"] = R.kcore()
        d["kcore_partitioned"] = R1.kcore(partitioned=True)
        d["mis"] = R.mis()
        d["cdlp"] = R.cdlp(np.arange(n, dtype=np.int32), 10)
        d["cdlp_partitioned"] = R.cdlp(np.arange(n, dtype=np.int32), 10, partitioned=True)
    R.close()
    R1.close()
    return d


def summary_rmat16():
    """Config-1 graph (RMAT-16 ef16 seed 1, 64 equal partitions): scalars and
    checksums only, to keep the fixture small."""
    h = pc.HostCSR.rmat(16, 16, 1).add_weights(seed=1, wmax=255)
    vl, el, w = h.arrays()
    n = vl.size - 1
    R = O.Reference(vl, el, w=w, v2p=pc.equal_vertex_partition(n, 64))
    R1 = O.Reference(vl, el, w=w, v2p=pc.equal_vertex_partition(n, 64), threads=1)
    lev = levels_from_parents(R.bfs_parents(0), 0)
    core = R.kcore()
    mis = R.mis()
    cd = R.cdlp(np.arange(n, dtype=np.int32), 10)
    lcc = R.lcc()
    sssp = R1.sssp(0, partitioned=True)  # exact distances (see test_oracle.py)
    pr = R.pagerank(0.85, 20, partitioned=True)
    s = {
        "n": int(n), "m": int(el.size),
        "tc_merge": R.tc(), "tc_merge_partitioned": R.tc(partitioned=True),
        "tc_galloping": R.tc(galloping=True),
        "bfs_levels_sum": int(lev[lev < 2**31 - 1].astype(np.int64).sum()),
        "bfs_unreached": int((lev == 2**31 - 1).sum()),
        "kcore_sum": int(core.astype(np.int64).sum()), "kcore_max": int(core.max()),
        "mis_size": int(mis.sum()), "mis_index_sum": int(np.nonzero(mis)[0].astype(np.int64).sum()),
        "cdlp_sum": int(cd.astype(np.int64).sum()),
        "lcc_nan": int(np.isnan(lcc).sum()), "lcc_sum": float(np.nansum(lcc)),
        "sssp_sum": int(sssp[sssp < 2**31 // 2].astype(np.int64).sum()),
        "pagerank_f32_sum": float(pr.astype(np.float64).sum()), "pagerank_f32_max": float(pr.max()),
        "graph_checksum": int((vl.astype(np.uint64) * np.uint64(2654435761)).sum() % 2**61
                              + (el.astype(np.uint64) * np.uint64(40503)).sum() % 2**61),
    }
    R.close()
    R1.close()
    return s


def main():
    if not O.Reference.available():
        O.build(ref=True)
    for name, (vl, el, w), P in graphs():
        d = run_reference(name, vl, el, w, P)
        np.savez_compressed(OUT / f"{name}.npz", **{k: np.asarray(v) for k, v in d.items()})
        print("wrote", name, int(d["tc_merge"]))
    s = summary_rmat16()
    (OUT / "rmat16_summary.json").write_text(json.dumps(s, indent=1) + "\n")
    print("wrote rmat16_summary.json", s["tc_merge"])


if __name__ == "__main__":
    main()
