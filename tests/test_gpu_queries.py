"""Multi-way queries on the GPU (pc_friend_triangle, pc_square_count)
against the reference's own outputs (golden fixtures) and the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN_GRAPHS, load_golden
from test_oracle import partition_contiguous_ids, relabel_csr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", GOLDEN_GRAPHS)
def test_queries_match_golden(gpu, name):
    pc = gpu
    d = load_golden(name)
    if "friend_root" not in d:
        pytest.skip("no queries for this graph")
    g = pc.Graph(vlist=d["vlist"], elist=d["elist"])
    pg = pc.Partitioned_Graph(g, d["v2p"])
    assert pg.solve_friend_triangle_merge(int(d["friend_root"]), d["friend_nodes"]) == int(d["friend_partitioned"])
    assert pg.solve_friend_triangle_galloping(int(d["friend_root"]), d["friend_nodes"]) == \
        int(d["friend_partitioned_galloping"])
    assert g.solve_friend_triangle_merge(int(d["friend_root"]), d["friend_nodes"]) == int(d["friend_merge"])
    assert pg.solve_square_counting() == int(d["squares_partitioned"])
    pg.close()
    g.close()


@pytest.mark.parametrize("scale,seed", [(12, 3), (16, 1)])
def test_queries_match_oracle_with_reorder(gpu, O, scale, seed):
    pc = gpu
    vl, el, _ = pc.HostCSR.rmat(scale, 16, seed).arrays()
    n = vl.size - 1
    rng = np.random.default_rng(seed)
    v2p = rng.integers(0, 9, n).astype(np.int32)  # non-contiguous partitions
    g = pc.Graph(vlist=vl, elist=el)
    pg = pc.Partitioned_Graph(g, v2p)
    nodes = rng.integers(0, n, 300).astype(np.int32)
    nodes[7] = 0
    assert pg.solve_friend_triangle_merge(0, nodes) == O.friend_triangle(vl, el, 0, nodes)
    assert pg.solve_friend_triangle_merge(n - 1, nodes[:2]) == O.friend_triangle(vl, el, n - 1, nodes[:2])
    assert pg.solve_friend_triangle_merge(3, nodes[:1]) == 0
    sq = O.square_count(vl, el)
    assert pg.solve_square_counting() == sq
    # after reorder() the ids are the partition-contiguous ones; squares depend on the order
    pg.reorder()
    o2n = partition_contiguous_ids(v2p)
    nvl, nel = relabel_csr(vl, el, o2n)
    assert pg.solve_square_counting() == O.square_count(nvl, nel)
    assert pg.solve_friend_triangle_merge(int(o2n[0]), o2n[nodes].astype(np.int32)) == \
        O.friend_triangle(vl, el, 0, nodes)
    pg.close()
    g.close()


def test_queries_reject_bad_ids(gpu):
    pc = gpu
    d = load_golden("tiny")
    g = pc.Graph(vlist=d["vlist"], elist=d["elist"])
    pg = pc.Partitioned_Graph(g, d["v2p"])
    with pytest.raises(pc.PCError):
        pg.solve_friend_triangle_merge(9, [0, 1])
    with pytest.raises(pc.PCError):
        pg.solve_friend_triangle_merge(0, [1, 7])
    pg.close()
    g.close()
