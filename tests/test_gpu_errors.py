"""Malformed inputs are rejected with PC_ERR_INVALID_INPUT by the device-side
validation and the argument checks, and the library stays usable after an
error (no fault, no hang: every check is a bounded kernel or a host test)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import csr_from_edges

pytestmark = pytest.mark.gpu


def _raises_invalid(fn):
    import partitionandconquer_b200 as pc
    with pytest.raises(pc.PCError) as e:
        fn()
    assert e.value.status == 1, str(e.value)
    return str(e.value)


def test_rejects_malformed_csr(gpu):
    pc = gpu
    vl, el = csr_from_edges(5, [(0, 1), (1, 2), (2, 3), (3, 4), (0, 2)])
    # asymmetric: drop one direction of an edge
    bad_el = el.copy()
    bad_vl = vl.copy()
    row0 = bad_el[bad_vl[0]:bad_vl[1]]
    assert row0.tolist() == [1, 2]
    asym_el = np.delete(bad_el, 1)
    asym_vl = bad_vl.copy()
    asym_vl[1:] -= 1
    msg = _raises_invalid(lambda: pc.Graph(vlist=asym_vl, elist=asym_el)._device())
    assert "symmetric" in msg
    # unsorted row
    uns = el.copy()
    uns[vl[0]], uns[vl[0] + 1] = uns[vl[0] + 1], uns[vl[0]]
    assert "ascending" in _raises_invalid(lambda: pc.Graph(vlist=vl, elist=uns)._device())
    # self-loop
    vl2, el2 = csr_from_edges(3, [(0, 1)])
    sl_el = np.array([0, 1, 0], np.int32)
    sl_vl = np.array([0, 2, 3, 3], np.uint64)
    assert "self-loop" in _raises_invalid(lambda: pc.Graph(vlist=sl_vl, elist=sl_el)._device())
    # out of range id
    oor = el.copy()
    oor[-1] = 99
    assert "outside" in _raises_invalid(lambda: pc.Graph(vlist=vl, elist=oor)._device())
    # non-monotone offsets
    nm = vl.copy()
    nm[2], nm[3] = nm[3], nm[2]
    _raises_invalid(lambda: pc.Graph(vlist=nm, elist=el)._device())
    # the device is still fine
    g = pc.Graph(vlist=vl, elist=el)
    assert g.solve_triangle_counting_merge() == 1


def test_rejects_bad_arguments(gpu):
    pc = gpu
    vl, el = csr_from_edges(6, [(0, 1), (1, 2), (2, 0), (3, 4)])
    g = pc.Graph(vlist=vl, elist=el, weights=np.ones(el.size, np.int32))
    _raises_invalid(lambda: pc.Partitioned_Graph(g, np.array([0, 1, -1, 0, 0, 0], np.int32)))
    pg = pc.Partitioned_Graph(g, np.array([0, 0, 1, 1, 2, 2], np.int32))
    _raises_invalid(lambda: pg.solve_bfs(6))
    _raises_invalid(lambda: pg.solve_bfs(-1))
    _raises_invalid(lambda: pg.solve_sssp(7))
    _raises_invalid(lambda: pg.solve_sssp(0, method=3))
    _raises_invalid(lambda: pg.solve_sssp(0, method=pc.SSSP_DELTA_STEPPING, delta=-1))
    _raises_invalid(lambda: pg.batch_cnt_common_neis_merge(np.array([[0, 9]], np.int32)))
    _raises_invalid(lambda: pg.jaccard_queries(np.array([0, 6], np.int32)))
    _raises_invalid(lambda: pg.page_rank(0.85, 0))
    _raises_invalid(lambda: pg.page_rank(1.5, 3))
    _raises_invalid(lambda: pg.triangle_count(variant=17))
    unweighted = pc.Partitioned_Graph(pc.Graph(vlist=vl, elist=el), None)
    assert "weighted" in _raises_invalid(lambda: unweighted.solve_sssp(0))
    assert pg.solve_triangle_counting_merge() == 1


def test_empty_and_tiny_graphs(gpu, O):
    pc = gpu
    for n in (1, 2, 5):
        vl = np.zeros(n + 1, np.uint64)
        el = np.zeros(0, np.int32)
        g = pc.Graph(vlist=vl, elist=el, weights=el)
        pg = pc.Partitioned_Graph(g, np.zeros(n, np.int32))
        assert pg.solve_triangle_counting_merge() == 0
        assert pg.solve_bfs(0).tolist() == [-1] + [2**31 - 1] * (n - 1)
        assert pg.solve_sssp(0).tolist() == [0] + [(2**31 - 1) // 2] * (n - 1)
        np.testing.assert_array_equal(pg.solve_sssp(0), O.sssp(vl, el, el, 0))
        assert pg.solve_kcore().tolist() == [0] * n
        assert pg.solve_mis().tolist() == [1] * n
        np.testing.assert_array_equal(pg.solve_lcc_merge(), np.zeros(n))
        pr = pg.page_rank(0.85, 3, fp64=True)
        np.testing.assert_allclose(pr, np.full(n, 0.15 / n), rtol=1e-15)
    # a complete graph: the reference's peeling stops at level n-1 and leaves 0
    vl, el = csr_from_edges(6, [(i, j) for i in range(6) for j in range(i + 1, 6)])
    pg = pc.Partitioned_Graph(pc.Graph(vlist=vl, elist=el), None)
    assert pg.solve_kcore().tolist() == [0] * 6
    assert pg.solve_triangle_counting_merge() == 20


def test_rejects_bad_weights(gpu):
    pc = gpu
    vl, el = csr_from_edges(4, [(0, 1), (1, 2), (2, 3)])
    w = np.ones(el.size, np.int32)
    w[0] = -1
    assert "weights" in _raises_invalid(lambda: pc.Graph(vlist=vl, elist=el, weights=w)._device())
    w[0] = 1 << 30
    _raises_invalid(lambda: pc.Graph(vlist=vl, elist=el, weights=w)._device())


def test_grid_barrier_is_bounded(gpu):
    """The persistent kernels' grid barrier orders every CTA, and a CTA that
    never arrives makes the others' waits run out (a short limit) into a
    TIMEOUT status, leaving the device usable."""
    pc = gpu
    assert pc.selftest_grid_barrier(0, rounds=200) == 0
    with pytest.raises(pc.PCError) as e:
        pc.selftest_grid_barrier(0, rounds=4, absent_cta=3, limit_ms=100)
    assert "ran out of time" in str(e.value)
    assert pc.selftest_grid_barrier(0, rounds=8) == 0
    h = pc.HostCSR.rmat(10, 8, 3)
    vl, el, _ = h.arrays()
    g = pc.Graph(vlist=vl, elist=el)
    pg = pc.Partitioned_Graph(g, pc.equal_vertex_partition(vl.size - 1, 4))
    from oracle import oracle as O
    np.testing.assert_array_equal(pg.solve_kcore(), O.kcore(vl, el)[0])
    pg.close()
    g.close()
