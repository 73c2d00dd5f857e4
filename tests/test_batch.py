"""Many graphs in one launch (pc_batch_*): the seeded arena generator on the
CPU; per-graph TC, LCC and BFS against the oracle on the GPU, across every
schedule, with the captured CUDA graph replayed."""
from __future__ import annotations

import numpy as np
import pytest


def graph_slice(vl, el, voff, g):
    v0, v1 = int(voff[g]), int(voff[g + 1])
    sub_vl = (vl[v0:v1 + 1] - vl[v0]).astype(np.uint64)
    sub_el = (el[vl[v0]:vl[v1]] - v0).astype(np.int32)
    return sub_vl, sub_el


def test_batch_arena_generator(pc):
    h, voff = pc.HostCSR.rmat_batch(24, 5, 9, 4, 12, seed=3)
    vl, el, _ = h.arrays()
    h2, voff2 = pc.HostCSR.rmat_batch(24, 5, 9, 4, 12, seed=3)
    np.testing.assert_array_equal(voff, voff2)
    np.testing.assert_array_equal(el, h2.arrays()[1])
    sizes = np.diff(voff)
    assert sizes.min() >= 32 and sizes.max() <= 512 and np.all((sizes & (sizes - 1)) == 0)
    for g in range(24):
        sv, se = graph_slice(vl, el, voff, g)
        n = sv.size - 1
        assert se.size == 0 or (se.min() >= 0 and se.max() < n)  # no edge leaves the graph
        # graph g is the standalone generator's graph with seed g
        scale = int(np.log2(n))
        found = False
        for ef in range(4, 13):
            v2, e2, _ = pc.HostCSR.rmat(scale, ef, g).arrays()
            if v2.size == sv.size and e2.size == se.size and np.array_equal(v2, sv) and np.array_equal(e2, se):
                found = True
                break
        assert found, g


@pytest.mark.gpu
def test_batch_matches_oracle_every_schedule(gpu, O):
    pc = gpu
    h, voff = pc.HostCSR.rmat_batch(40, 6, 11, 4, 16, seed=1)
    vl, el, _ = h.arrays()
    G = voff.size - 1
    exp_tc = np.zeros(G, np.uint64)
    exp_lcc = np.zeros(vl.size - 1)
    exp_bfs = np.zeros(vl.size - 1, np.int32)
    for g in range(G):
        sv, se = graph_slice(vl, el, voff, g)
        v0, v1 = int(voff[g]), int(voff[g + 1])
        exp_tc[g] = O.tc_merge(sv, se)
        exp_lcc[v0:v1] = O.lcc(sv, se)
        exp_bfs[v0:v1] = O.bfs(sv, se, 0)
    b = pc.Batch(vl, el, voff)
    for threads, cps, order in [(512, 2, 0), (256, 4, 1), (256, 1, 0), (512, 1, 1)]:
        b.set_schedule(threads, cps, order)
        for _ in range(2):  # the second run replays the captured graph
            r = b.run()
            np.testing.assert_array_equal(r["tc"], exp_tc)
            np.testing.assert_array_equal(np.isnan(r["lcc"]), np.isnan(exp_lcc))
            np.testing.assert_array_equal(r["lcc"], exp_lcc)
            np.testing.assert_array_equal(r["bfs"], exp_bfs)
            assert r["items"] == 3 * G and r["ms"] > 0
    only_tc = b.run(pc.Batch.TC)
    np.testing.assert_array_equal(only_tc["tc"], exp_tc)
    assert only_tc["lcc"] is None and only_tc["items"] == G
    best = b.autotune()
    assert best["threads"] in (256, 512) and best["ms"] > 0
    np.testing.assert_array_equal(b.run()["tc"], exp_tc)
    b.close()


@pytest.mark.gpu
def test_batch_rejects_edges_between_graphs(gpu):
    pc = gpu
    from conftest import csr_from_edges
    vl, el = csr_from_edges(6, [(0, 1), (1, 2), (2, 3), (3, 4)])  # 2-3 crosses the split at 3
    with pytest.raises(pc.PCError) as e:
        pc.Batch(vl, el, np.array([0, 3, 6], np.uint64))
    assert "joins two graphs" in str(e.value)
