"""Ingest on the device (pc_graph_from_edges / pc_graph_rmat / pc_graph_er /
pc_graph_add_weights): the CSR built by radix sort + unique on the GPU must
equal, bit for bit, the host builders' arrays and an independent numpy
restatement of the text loader's adjacency build (src/Graph.cpp:59-85)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def numpy_csr(src, dst, n):
    """Both directions, self-loops dropped, rows sorted and deduplicated."""
    s = np.asarray(src, np.int64)
    d = np.asarray(dst, np.int64)
    keep = s != d
    u = np.concatenate([s[keep], d[keep]])
    v = np.concatenate([d[keep], s[keep]])
    key = np.unique(u * n + v)
    rows, cols = key // n, key % n
    vl = np.zeros(n + 1, np.uint64)
    np.cumsum(np.bincount(rows, minlength=n), out=vl[1:])
    return vl, cols.astype(np.int32)


def numpy_relabel(vl, el):
    n = vl.size - 1
    deg = np.diff(vl).astype(np.int64)
    new2old = np.lexsort((np.arange(n), -deg))
    old2new = np.empty(n, np.int64)
    old2new[new2old] = np.arange(n)
    rows = np.repeat(np.arange(n), deg)
    key = np.sort(old2new[rows] * n + old2new[el.astype(np.int64)])
    nvl = np.zeros(n + 1, np.uint64)
    np.cumsum(np.bincount(key // n, minlength=n), out=nvl[1:])
    return nvl, (key % n).astype(np.int32), old2new.astype(np.int32)


@pytest.mark.parametrize("n,ne,seed", [(1, 3, 0), (7, 40, 1), (300, 5000, 2), (1 << 14, 200000, 3)])
def test_from_edges_matches_numpy(gpu, n, ne, seed):
    pc = gpu
    rng = np.random.default_rng(seed)
    src = rng.integers(0, n, ne).astype(np.uint32)
    dst = rng.integers(0, n, ne).astype(np.uint32)
    k = ne // 8
    if k:
        src[:k] = dst[:k]                                   # self-loops
        src[-k:], dst[-k:] = dst[k:2 * k], src[k:2 * k]     # reversed repeats
        src[-2 * k:-k], dst[-2 * k:-k] = src[k:2 * k], dst[k:2 * k]  # exact repeats
    vl, el = numpy_csr(src, dst, n)
    g = pc.Graph.from_edges(src, dst, n, relabel=False)
    np.testing.assert_array_equal(g.get_csr_vlist(), vl)
    np.testing.assert_array_equal(g.get_csr_elist(), el)
    g.close()
    rvl, rel, o2n = numpy_relabel(vl, el)
    g2, m2 = pc.Graph.from_edges(src, dst, n, relabel=True, return_map=True)
    np.testing.assert_array_equal(g2.get_csr_vlist(), rvl)
    np.testing.assert_array_equal(g2.get_csr_elist(), rel)
    np.testing.assert_array_equal(m2, o2n)
    g2.close()


def test_from_edges_empty_and_isolated(gpu):
    pc = gpu
    g = pc.Graph.from_edges(np.zeros(0, np.uint32), np.zeros(0, np.uint32), 5, relabel=True)
    np.testing.assert_array_equal(g.get_csr_vlist(), np.zeros(6, np.uint64))
    assert g.get_edge_num() == 0
    g.close()
    g = pc.Graph.from_edges(np.array([3, 3], np.uint32), np.array([1, 3], np.uint32), 6, relabel=False)
    np.testing.assert_array_equal(g.get_csr_vlist(), np.array([0, 0, 1, 1, 2, 2, 2], np.uint64))
    np.testing.assert_array_equal(g.get_csr_elist(), np.array([3, 1], np.int32))
    g.close()


def test_from_edges_rejects_out_of_range(gpu):
    pc = gpu
    with pytest.raises(pc.PCError) as e:
        pc.Graph.from_edges(np.array([0, 9], np.uint32), np.array([1, 2], np.uint32), 5)
    assert "outside" in str(e.value)


@pytest.mark.parametrize("scale,ef,seed", [(10, 16, 1), (16, 16, 1), (20, 8, 5)])
def test_device_rmat_equals_host_generator(gpu, scale, ef, seed):
    pc = gpu
    h = pc.HostCSR.rmat(scale, ef, seed)
    vl, el, _ = h.arrays()
    g = pc.Graph.rmat_device(scale, ef, seed)
    np.testing.assert_array_equal(g.get_csr_vlist(), vl)
    np.testing.assert_array_equal(g.get_csr_elist(), el)
    g.close()
    hr = pc.HostCSR.rmat(scale, ef, seed, relabel=False)
    g = pc.Graph.rmat_device(scale, ef, seed, relabel=False)
    np.testing.assert_array_equal(g.get_csr_elist(), hr.arrays()[1])
    g.close()


def test_device_er_and_weights_equal_host(gpu):
    pc = gpu
    h = pc.HostCSR.er(14, 1 << 18, 4)
    g = pc.Graph.er_device(14, 1 << 18, 4)
    np.testing.assert_array_equal(g.get_csr_vlist(), h.arrays()[0])
    np.testing.assert_array_equal(g.get_csr_elist(), h.arrays()[1])
    g.close()
    h = pc.HostCSR.rmat(12, 16, 2)
    h.add_weights(seed=9, wmax=255)
    g = pc.Graph.rmat_device(12, 16, 2, wmax=255, weight_seed=9)
    np.testing.assert_array_equal(g.get_csr_weight(), h.arrays()[2])
    g.close()


def test_device_built_graph_runs_the_algorithms(gpu, O):
    pc = gpu
    g = pc.Graph.rmat_device(13, 16, 7)
    vl, el = g.get_csr_vlist(), g.get_csr_elist()
    pg = pc.Partitioned_Graph(g, pc.equal_vertex_partition(vl.size - 1, 16))
    assert pg.solve_triangle_counting_merge() == O.tc_merge(vl, el)
    np.testing.assert_array_equal(pg.solve_bfs(0), O.bfs(vl, el, 0))
    pg.close()
    g.close()


@pytest.mark.parametrize("one_based", [0, 1])
def test_cli_preprocess_on_device_matches_reference_tool(gpu, tmp_path, one_based):
    """`pc_main preprocess` builds the adjacency on the GPU when one is
    present; its files must equal the reference preprocess tool's bytes."""
    import subprocess

    from test_cli_host import PC_MAIN, REF_PRE, write_edge_list
    if not PC_MAIN.exists() or not REF_PRE.exists():
        pytest.skip("pc_main or the reference preprocess tool is not built")
    for tool, d in ((str(PC_MAIN), tmp_path / "ours"), (str(REF_PRE), tmp_path / "ref")):
        (d / "origin").mkdir(parents=True)
        write_edge_list(d / "graph.txt", np.random.default_rng(20 + one_based), 2000, 30000, one_based)
        args = [tool, "preprocess", str(d) + "/", "graph.txt"] if tool == str(PC_MAIN) else [tool, str(d) + "/", "graph.txt"]
        r = subprocess.run(args, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
    for f in ("csr_vlist.bin", "csr_elist.bin", "csr_weight.bin"):
        assert (tmp_path / "ours" / "origin" / f).read_bytes() == (tmp_path / "ref" / "origin" / f).read_bytes(), f
