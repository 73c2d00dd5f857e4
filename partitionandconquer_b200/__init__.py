"""B200-native partitioned-CSR graph analytics (the hot path of PartitionAndConquer).

Python mirror of the reference's host API -- ``Graph`` and
``Partitioned_Graph`` of src/Graph.hpp -- over the C ABI of libpc.so
(include/pc.h).  Method names, argument meaning and result conventions follow
the reference; results come back as numpy arrays instead of filling
``std::vector`` out-parameters.  All computation runs in hand-written sm_100a
kernels; there is no CPU fallback (a missing GPU raises PCError).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import (METHOD_GALLOPING, METHOD_MERGE, NUM_VARIANTS, VARIANT_AUTO, VARIANT_HEURISTIC, VARIANTS,
                   PCError, TCStats, check, lib, ptr)

__all__ = [
    "Graph", "Partitioned_Graph", "HostCSR", "PCError", "TCStats", "VARIANTS", "VARIANT_AUTO",
    "VARIANT_HEURISTIC", "equal_vertex_partition", "device_count", "launch_count", "selector", "Batch",
]

INT_MAX = 2**31 - 1
INGEST_DEGREE_RELABEL = 1  # PC_INGEST_DEGREE_RELABEL


def device_count() -> int:
    return int(lib.pc_device_count())


SSSP_AUTO, SSSP_BELLMAN_FORD, SSSP_DELTA_STEPPING = 0, 1, 2


def launch_count() -> int:
    """Kernels launched by libpc.so in this process."""
    return int(lib.pc_launch_count())


def selftest_grid_barrier(device: int = 0, rounds: int = 64, absent_cta: int = -1, limit_ms: int = 1000) -> int:
    """Runs the bounded grid barrier of the persistent kernels `rounds` times
    and returns the number of ordering violations seen (0 expected).  With
    absent_cta >= 0 one CTA never arrives and PCError (status TIMEOUT) is
    raised once the others' waits run out."""
    bad = C.c_uint32(0)
    check(lib.pc_selftest_grid_barrier(device, rounds, absent_cta, limit_ms, C.byref(bad)))
    return int(bad.value)


def vertex_priority(seed: int, n: int) -> np.ndarray:
    """Priorities Partitioned_Graph.solve_mis(seed=...) orders vertices by."""
    out = np.empty(n, np.uint64)
    check(lib.pc_synth_vertex_priority(seed, n, ptr(out)))
    return out


def _result(out, size: int, dtype) -> np.ndarray:
    """The array a call writes its result into: a new one, or the caller's
    `out`, which must be a writeable C-contiguous array of `size` entries of
    `dtype`.  Page-locked memory (a pinned torch tensor's .numpy(), or an
    array registered with pc_host_register) lets the copy back run at DMA
    speed; a new pageable array is faulted in by the copy itself."""
    if out is None:
        return np.empty(size, dtype)
    if (not isinstance(out, np.ndarray) or out.dtype != np.dtype(dtype) or out.size != size
            or not out.flags.c_contiguous or not out.flags.writeable):
        raise ValueError(f"out must be a writeable C-contiguous {np.dtype(dtype).name} array of {size} entries")
    return out


def equal_vertex_partition(n: int, P: int) -> np.ndarray:
    """part(u) = floor(u * P / n): P contiguous blocks of equal vertex count."""
    return ((np.arange(n, dtype=np.int64) * P) // max(n, 1)).astype(np.int32)


class HostCSR:
    """Host CSR in the reference's binary format, from the seeded generators or files."""

    def __init__(self, handle):
        self._h = handle

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:  # at interpreter exit the module may be torn down first
            lib.pc_host_csr_free(h)
            self._h = None

    @classmethod
    def _make(cls, fn, *args):
        out = C.c_void_p()
        check(fn(*args, C.byref(out)))
        return cls(out)

    @classmethod
    def rmat(cls, scale: int, edge_factor: int = 16, seed: int = 1, relabel: bool = True) -> "HostCSR":
        """RMAT(0.57, 0.19, 0.19, 0.05) symmetrised, deduplicated, degree-relabelled."""
        return cls._make(lib.pc_synth_rmat, scale, edge_factor, seed, int(relabel))

    @classmethod
    def er(cls, scale: int, nedges: int, seed: int = 1, relabel: bool = True) -> "HostCSR":
        return cls._make(lib.pc_synth_er, scale, nedges, seed, int(relabel))

    @classmethod
    def chung_lu(cls, scale: int, nedges: int, beta: float = 2.1, dmax: int = 1 << 20, seed: int = 1,
                 relabel: bool = True) -> "HostCSR":
        return cls._make(lib.pc_synth_chung_lu, scale, nedges, beta, dmax, seed, int(relabel))

    @classmethod
    def load(cls, csrdir: str, weighted: bool = False) -> "HostCSR":
        return cls._make(lib.pc_host_csr_load, csrdir.encode(), int(weighted))

    @classmethod
    def from_arrays(cls, vlist, elist, weights=None) -> "HostCSR":
        vl = _lib.as_array(vlist, np.uint64)
        el = _lib.as_array(elist, np.int32)
        w = None if weights is None else _lib.as_array(weights, np.int32)
        return cls._make(lib.pc_host_csr_from_arrays, ptr(vl), ptr(el), ptr(w), vl.size - 1, el.size)

    @classmethod
    def rmat_batch(cls, G: int, smin: int = 10, smax: int = 16, emin: int = 8, emax: int = 32, seed: int = 0):
        """G seeded RMAT graphs in one arena; returns (HostCSR, voff[G+1])."""
        out = C.c_void_p()
        voff = np.zeros(G + 1, np.uint64)
        check(lib.pc_synth_rmat_batch(G, smin, smax, emin, emax, seed, C.byref(out), ptr(voff)))
        return cls(out), voff

    def add_weights(self, seed: int = 1, wmax: int = 255) -> "HostCSR":
        check(lib.pc_synth_add_weights(self._h, seed, wmax))
        return self

    def save(self, csrdir: str):
        os.makedirs(csrdir, exist_ok=True)
        check(lib.pc_host_csr_save(self._h, csrdir.encode()))

    def arrays(self, copy: bool = True):
        """(vlist uint64[n+1], elist int32[m], weights int32[m] or None)."""
        n, m = C.c_uint64(), C.c_uint64()
        vl, el, w = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(lib.pc_host_csr_arrays(self._h, C.byref(n), C.byref(m), C.byref(vl), C.byref(el), C.byref(w)))
        nn, mm = n.value, m.value

        def view(p, count, dt):
            if count == 0 or not p.value:
                return np.zeros(count, dt)
            buf = (C.c_char * (count * np.dtype(dt).itemsize)).from_address(p.value)
            a = np.frombuffer(buf, dtype=dt, count=count)
            return a.copy() if copy else a

        vlist = view(vl, nn + 1, np.uint64)
        elist = view(el, mm, np.int32)
        weights = view(w, mm, np.int32) if w.value else None
        return vlist, elist, weights


class Graph:
    """Mirror of ``class Graph`` (src/Graph.hpp:38-103).

    Construct from a CSR directory (``Graph(csrdir, is_weighted)``, the binary
    files of src/Graph.cpp:92-137), from arrays, or from an adjacency list
    (src/Graph.cpp:139-149).  The CSR is uploaded to the GPU on first use; the
    ``solve_*`` methods run the unpartitioned algorithms (one partition).
    """

    def __init__(self, csrdir: Optional[str] = None, is_weighted: bool = False, *, vlist=None, elist=None,
                 weights=None, adj_list: Optional[Sequence[Sequence[int]]] = None, host: Optional[HostCSR] = None,
                 validate: bool = True):
        if host is not None:
            vlist, elist, weights = host.arrays()
        elif csrdir is not None:
            vlist, elist, weights = HostCSR.load(csrdir, is_weighted).arrays()
        elif adj_list is not None:
            lens = np.array([len(a) for a in adj_list], dtype=np.uint64)
            vlist = np.zeros(len(adj_list) + 1, np.uint64)
            np.cumsum(lens, out=vlist[1:])
            elist = np.concatenate([np.asarray(a, np.int32) for a in adj_list]) if len(adj_list) else np.zeros(0, np.int32)
        if vlist is None or elist is None:
            raise ValueError("Graph needs a csrdir, arrays, an adjacency list or a HostCSR")
        self.vlist = _lib.as_array(vlist, np.uint64)
        self.elist = _lib.as_array(elist, np.int32)
        self.weights = None if weights is None else _lib.as_array(weights, np.int32)
        self.validate = validate
        self._g = None
        self._pg = None

    # -- built on the device (pc_graph_from_edges / pc_graph_rmat / pc_graph_er) --
    @classmethod
    def _adopt(cls, handle) -> "Graph":
        """Wraps a device-built handle; the host arrays are downloaded once."""
        n, m, w = C.c_uint64(), C.c_uint64(), C.c_int32()
        check(lib.pc_graph_info(handle, C.byref(n), C.byref(m), C.byref(w)))
        vl = np.empty(n.value + 1, np.uint64)
        el = np.empty(m.value, np.int32)
        wt = np.empty(m.value, np.int32) if w.value else None
        check(lib.pc_graph_download(handle, ptr(vl), ptr(el), ptr(wt)))
        obj = cls.__new__(cls)
        obj.vlist, obj.elist, obj.weights = vl, el, wt
        obj.validate = False
        obj._g = handle
        obj._pg = None
        return obj

    @classmethod
    def from_edges(cls, src, dst, n: int, relabel: bool = True, return_map: bool = False):
        """Symmetric, deduplicated CSR built on the GPU from a raw edge stream
        (the text loader's adjacency build, src/Graph.cpp:59-85)."""
        s = _lib.as_array(src, np.uint32)
        d = _lib.as_array(dst, np.uint32)
        if s.size != d.size:
            raise ValueError("src and dst must have the same length")
        o2n = np.empty(n, np.int32) if (relabel and return_map) else None
        out = C.c_void_p()
        check(lib.pc_graph_from_edges(ptr(s), ptr(d), s.size, n, INGEST_DEGREE_RELABEL if relabel else 0, ptr(o2n),
                                      C.byref(out)))
        g = cls._adopt(out)
        return (g, o2n) if return_map else g

    @classmethod
    def rmat_device(cls, scale: int, edge_factor: int = 16, seed: int = 1, relabel: bool = True, wmax: int = 0,
                    weight_seed: int = 1) -> "Graph":
        """HostCSR.rmat's graph, generated and built on the GPU."""
        out = C.c_void_p()
        check(lib.pc_graph_rmat(scale, edge_factor, seed, INGEST_DEGREE_RELABEL if relabel else 0, C.byref(out)))
        if wmax:
            try:
                check(lib.pc_graph_add_weights(out, weight_seed, wmax))
            except Exception:
                lib.pc_graph_destroy(out)
                raise
        return cls._adopt(out)

    @classmethod
    def er_device(cls, scale: int, nedges: int, seed: int = 1, relabel: bool = True) -> "Graph":
        """HostCSR.er's graph, generated and built on the GPU."""
        out = C.c_void_p()
        check(lib.pc_graph_er(scale, nedges, seed, INGEST_DEGREE_RELABEL if relabel else 0, C.byref(out)))
        return cls._adopt(out)

    # -- accessors (src/Graph.cpp:151-307) --
    def get_vertex_num(self) -> int:
        return int(self.vlist.size - 1)

    def get_edge_num(self) -> int:
        return int(self.elist.size)

    def is_weighted(self) -> bool:
        return self.weights is not None

    def get_csr_vlist(self):
        return self.vlist

    def get_csr_elist(self):
        return self.elist

    def get_csr_weight(self):
        return self.weights

    def get_deg(self, u: int) -> int:
        return int(self.vlist[u + 1] - self.vlist[u])

    def get_degs(self):
        return np.diff(self.vlist).astype(np.int32)

    def get_max_deg(self) -> int:
        return int(np.diff(self.vlist).max()) if self.vlist.size > 1 else 0

    def get_neis(self, u: int):
        return self.elist[self.vlist[u]:self.vlist[u + 1]].copy()

    def has_directed_edge(self, u: int, v: int) -> bool:
        row = self.elist[self.vlist[u]:self.vlist[u + 1]]
        i = np.searchsorted(row, v)
        return bool(i < row.size and row[i] == v)

    def has_edge(self, u: int, v: int) -> bool:
        return self.has_directed_edge(u, v) if self.get_deg(u) < self.get_deg(v) else self.has_directed_edge(v, u)

    def save_as_csr_binfile(self, csr_vlist_binfile: str, csr_elist_binfile: str):
        self.vlist.tofile(csr_vlist_binfile)
        self.elist.tofile(csr_elist_binfile)

    def random_partition(self, partition_num: int, seed: int = 1) -> np.ndarray:
        """Seeded stand-in for Graph::random_partition (src/Graph.cpp:564-570, which uses rand())."""
        rng = np.random.default_rng(seed)
        return rng.integers(0, partition_num, self.get_vertex_num(), dtype=np.int32)

    def greedy_partition(self, partition_num: int, seed: int = 1, on_device: bool = True) -> np.ndarray:
        """Graph::greedy_partition (src/Graph.cpp:898-967), seeded.  on_device:
        the GPU form (pc_greedy_partition); otherwise the sequential host rule."""
        out = np.empty(self.get_vertex_num(), np.int32)
        if on_device:
            check(lib.pc_greedy_partition(self._device(), partition_num, seed, ptr(out)))
        else:
            check(lib.pc_host_greedy_partition(ptr(self.vlist), ptr(self.elist), self.get_vertex_num(), partition_num,
                                               seed, ptr(out)))
        return out

    # -- device handles --
    def _device(self):
        if self._g is None:
            out = C.c_void_p()
            flags = 0 if self.validate else 1
            check(lib.pc_graph_create(ptr(self.vlist), ptr(self.elist), ptr(self.weights), self.vlist.size - 1,
                                      self.elist.size, flags, C.byref(out)))
            self._g = out
        return self._g

    def _one_partition(self):
        if self._pg is None:
            self._pg = Partitioned_Graph(self, None)
        return self._pg

    def stream(self) -> int:
        return int(lib.pc_graph_stream(self._device()) or 0)

    def close(self):
        if self._pg is not None:
            self._pg.close()
            self._pg = None
        if self._g is not None:
            lib.pc_graph_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- algorithms (unpartitioned Graph:: forms) --
    def solve_triangle_counting_merge(self, num_threads: int = 0) -> int:
        return self._one_partition().solve_triangle_counting_merge()

    def solve_triangle_counting_galloping(self, num_threads: int = 0) -> int:
        return self._one_partition().solve_triangle_counting_galloping()

    def solve_lcc_merge(self, num_threads: int = 0):
        return self._one_partition().solve_lcc_merge()

    def solve_lcc_galloping(self, num_threads: int = 0):
        return self._one_partition().solve_lcc_galloping()

    def solve_jsim_merge(self, queries, num_threads: int = 0):
        return self._one_partition().jaccard_queries(queries)

    solve_jsim_galloping = solve_jsim_merge

    def batch_cnt_common_neis_merge(self, queries, num_threads: int = 0):
        return self._one_partition().batch_cnt_common_neis_merge(queries)

    batch_cnt_common_neis_galloping = batch_cnt_common_neis_merge

    def solve_friend_triangle_merge(self, root: int, nodes, num_threads: int = 0) -> int:
        return self._one_partition().solve_friend_triangle_merge(root, nodes)

    solve_friend_triangle_galloping = solve_friend_triangle_merge

    def solve_bfs(self, u: int):
        """BFS levels from u (rank[u] = -1, unreached INT_MAX) -- the partitioned output convention."""
        return self._one_partition().solve_bfs(u)

    def solve_sssp(self, src: int):
        return self._one_partition().solve_sssp(src)

    def page_rank(self, pr_vals, damping_factor: float, num_iterations: int, num_threads: int = 0):
        """Graph::page_rank (src/Graph.cpp:534-554): starts from the caller's vector."""
        return self._one_partition().page_rank(damping_factor, num_iterations, init=pr_vals)

    def solve_kcore(self, num_threads: int = 0):
        return self._one_partition().solve_kcore()

    def solve_mis(self, num_threads: int = 0):
        return self._one_partition().solve_mis()

    def solve_cdlp(self, labels, max_iterations: int, num_threads: int = 0):
        return self._one_partition().solve_cdlp(labels, max_iterations)


class Partitioned_Graph:
    """Mirror of ``class Partitioned_Graph`` (src/Graph.hpp:105-155).

    ``Partitioned_Graph(g, vertex2partition, thread_num)``; ``thread_num`` is
    accepted for signature parity and ignored (the GPU schedules itself).
    ``vertex2partition=None`` means a single partition.
    """

    def __init__(self, g: Graph, vertex2partition=None, thread_num: int = 0):
        self.g = g
        gh = g._device()
        self.v2p = None if vertex2partition is None else _lib.as_array(vertex2partition, np.int32)
        if self.v2p is not None and self.v2p.size != g.get_vertex_num():
            raise ValueError("vertex2partition must have one entry per vertex")
        out = C.c_void_p()
        check(lib.pc_partition(gh, ptr(self.v2p), C.byref(out)))
        self._pg = out

    def close(self):
        if getattr(self, "_pg", None):
            lib.pc_pgraph_destroy(self._pg)
            self._pg = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._pg

    def get_vertex_num(self) -> int:
        return self.g.get_vertex_num()

    def get_edge_num(self) -> int:
        return self.g.get_edge_num()

    def get_partition_num(self) -> int:
        p = C.c_int32()
        check(lib.pc_pgraph_info(self._pg, None, None, C.byref(p)))
        return int(p.value)

    def reorder(self):
        check(lib.pc_pgraph_reorder(self._pg))

    def vertex_map(self):
        out = np.empty(self.get_vertex_num(), np.int32)
        check(lib.pc_pgraph_vertex_map(self._pg, ptr(out)))
        return out

    def layout(self):
        """(csr_vlist[P*n+1], csr_elist[m], csr_weight[m] or None) as the reference builds them."""
        n, P, m = self.get_vertex_num(), self.get_partition_num(), self.get_edge_num()
        vl = np.empty(P * n + 1, np.uint64)
        el = np.empty(m, np.int32)
        w = np.empty(m, np.int32) if self.g.is_weighted() else None
        check(lib.pc_pgraph_layout(self._pg, ptr(vl), ptr(el), ptr(w)))
        return vl, el, w

    def evaluate_partition(self):
        a, b, r = C.c_int64(), C.c_int64(), C.c_double()
        check(lib.pc_pgraph_evaluate(self._pg, C.byref(a), C.byref(b), C.byref(r)))
        return int(a.value), int(b.value), float(r.value)

    # -- intersection algorithms --
    def triangle_count(self, method: int = METHOD_MERGE, variant: int = VARIANT_AUTO, stats: bool = False):
        out = C.c_uint64()
        st = TCStats()
        check(lib.pc_tc_ex(self._pg, method, variant, C.byref(out), C.byref(st)))
        return (int(out.value), st) if stats else int(out.value)

    def solve_triangle_counting_merge(self) -> int:
        return self.triangle_count(METHOD_MERGE)

    def solve_triangle_counting_galloping(self) -> int:
        return self.triangle_count(METHOD_GALLOPING)

    def _lcc(self, method, out):
        out = _result(out, self.get_vertex_num(), np.float64)
        check(lib.pc_lcc(self._pg, method, ptr(out)))
        return out

    def solve_lcc_merge(self, out=None):
        return self._lcc(METHOD_MERGE, out)

    def solve_lcc_galloping(self, out=None):
        return self._lcc(METHOD_GALLOPING, out)

    def jaccard_edges(self, out=None):
        """J per CSR entry (fp32).  `out`, when given, is a C-contiguous float32
        host array of get_edge_num() entries that receives the values; pinned
        memory (e.g. a pinned torch tensor's .numpy()) makes the copy back run
        at DMA speed instead of being staged through the driver."""
        out = _result(out, self.get_edge_num(), np.float32)
        check(lib.pc_jaccard_edges(self._pg, ptr(out)))
        return out

    def jaccard_queries(self, queries):
        q = _lib.as_array(queries, np.int32)
        out = np.empty(q.size * q.size, np.float64)
        check(lib.pc_jaccard_queries(self._pg, ptr(q), q.size, ptr(out)))
        return out

    def solve_jsim_merge(self, queries):
        """J(q_i, q_j) = c / (d_i + d_j - c) -- the Graph:: formula (the partitioned reference
        version returns d_i + d_j - c without the division, src/Graph.cpp:2189-2194)."""
        return self.jaccard_queries(queries)

    solve_jsim_galloping = solve_jsim_merge

    def batch_cnt_common_neis_merge(self, queries):
        """queries: sequence of (u, v) pairs, or of vertex lists (k-sets)."""
        qs = list(queries) if not isinstance(queries, np.ndarray) else queries
        if isinstance(qs, np.ndarray) and qs.ndim == 2 and qs.shape[1] == 2:
            pairs = _lib.as_array(qs, np.int32).reshape(-1)
            out = np.empty(pairs.size // 2, np.uint64)
            check(lib.pc_batch_count_pairs(self._pg, ptr(pairs), pairs.size // 2, ptr(out)))
            return out
        if len(qs) and all(len(q) == 2 for q in qs):
            return self.batch_cnt_common_neis_merge(np.asarray(qs, np.int32).reshape(-1, 2))
        ids = np.concatenate([np.asarray(q, np.int32) for q in qs]) if len(qs) else np.zeros(0, np.int32)
        offs = np.zeros(len(qs) + 1, np.uint64)
        np.cumsum([len(q) for q in qs], out=offs[1:])
        out = np.empty(len(qs), np.uint64)
        check(lib.pc_batch_count_sets(self._pg, ptr(ids), ptr(offs), len(qs), ptr(out)))
        return out

    batch_cnt_common_neis_galloping = batch_cnt_common_neis_merge
    batch_cnt_common_neis_merge_fine_grained = batch_cnt_common_neis_merge

    def solve_friend_triangle_merge(self, root: int, nodes) -> int:
        """Sum over node pairs (positions j < k, the root skipped) of
        |N(root) & N(nodes[j]) & N(nodes[k])| (src/Graph.cpp:1222-1264)."""
        q = _lib.as_array(nodes, np.int32)
        out = C.c_uint64()
        check(lib.pc_friend_triangle(self._pg, int(root), ptr(q), q.size, C.byref(out)))
        return int(out.value)

    solve_friend_triangle_galloping = solve_friend_triangle_merge

    def solve_square_counting(self) -> int:
        """Partitioned_Graph::solve_square_counting (src/Graph.cpp:1291-1324)."""
        out = C.c_uint64()
        check(lib.pc_square_count(self._pg, C.byref(out)))
        return int(out.value)
    batch_cnt_common_neis_galloping_fine_grained = batch_cnt_common_neis_merge

    # -- frontier algorithms --
    # Every method below takes an optional `out`: a caller-owned host array
    # of the result's size and dtype that receives the result (see _result).
    def solve_bfs(self, u: int, out=None):
        out = _result(out, self.get_vertex_num(), np.int32)
        check(lib.pc_bfs(self._pg, u, ptr(out)))
        return out

    def solve_sssp(self, src: int, out=None, method: int = 0, delta: int = 0):
        """Exact distances from src.  method: SSSP_AUTO (0), SSSP_BELLMAN_FORD (1)
        or SSSP_DELTA_STEPPING (2) with bucket width `delta` (0: from the graph)."""
        out = _result(out, self.get_vertex_num(), np.int32)
        check(lib.pc_sssp_ex(self._pg, src, method, delta, ptr(out)))
        return out

    def page_rank(self, damping_factor: float = 0.85, num_iterations: int = 20, init=None, fp64: bool = False,
                  out=None):
        n = self.get_vertex_num()
        if fp64:
            out = _result(out, n, np.float64)
            ini = None if init is None else _lib.as_array(init, np.float64)
            check(lib.pc_pagerank_f64(self._pg, float(damping_factor), num_iterations, ptr(ini), ptr(out)))
        else:
            out = _result(out, n, np.float32)
            ini = None if init is None else _lib.as_array(init, np.float32)
            check(lib.pc_pagerank(self._pg, float(damping_factor), num_iterations, ptr(ini), ptr(out)))
        return out

    def solve_kcore(self, out=None):
        out = _result(out, self.get_vertex_num(), np.int32)
        largest = C.c_int32()
        check(lib.pc_kcore(self._pg, ptr(out), C.byref(largest)))
        return out

    def solve_mis(self, seed: Optional[int] = None, out=None):
        out = _result(out, self.get_vertex_num(), np.int32)
        if seed is None:
            check(lib.pc_mis(self._pg, ptr(out)))
        else:
            check(lib.pc_mis_hashed(self._pg, seed, ptr(out)))
        return out

    def solve_cdlp(self, labels, max_iterations: int, out=None):
        """Labels are updated in a copy (or in `out`); the input stays as it was."""
        lab = _lib.as_array(labels, np.int32)
        out = _result(out, self.get_vertex_num(), np.int32)
        if lab.size != out.size:
            raise ValueError(f"labels must have {out.size} entries")
        out[:] = lab
        check(lib.pc_cdlp(self._pg, max_iterations, ptr(out)))
        return out


class Batch:
    """Many independent graphs in one arena, processed in one persistent
    launch (pc_batch_* in include/pc.h).  Graph g owns arena vertices
    [voff[g], voff[g+1])."""

    TC, LCC, BFS = 1, 2, 4

    def __init__(self, vlist, elist, voff):
        self.vlist = _lib.as_array(vlist, np.uint64)
        self.elist = _lib.as_array(elist, np.int32)
        self.voff = _lib.as_array(voff, np.uint64)
        out = C.c_void_p()
        check(lib.pc_batch_create(ptr(self.vlist), ptr(self.elist), self.vlist.size - 1, self.elist.size,
                                  ptr(self.voff), self.voff.size - 1, C.byref(out)))
        self._b = out

    @property
    def num_graphs(self) -> int:
        return int(self.voff.size - 1)

    def run(self, tasks: int = 7):
        n = self.vlist.size - 1
        tc = np.zeros(self.num_graphs, np.uint64) if tasks & self.TC else None
        lcc = np.zeros(n, np.float64) if tasks & self.LCC else None
        bfs = np.zeros(n, np.int32) if tasks & self.BFS else None
        st = _lib.BatchStats()
        check(lib.pc_batch_run(self._b, tasks, ptr(tc), ptr(lcc), ptr(bfs), C.byref(st)))
        return {"tc": tc, "lcc": lcc, "bfs": bfs, "ms": st.ms, "items": st.items, "threads": st.threads,
                "ctas_per_sm": st.ctas_per_sm, "order": st.order}

    def set_schedule(self, threads: int = 512, ctas_per_sm: int = 2, order: int = 0):
        check(lib.pc_batch_set_schedule(self._b, threads, ctas_per_sm, order))

    def autotune(self, tasks: int = 7):
        st = _lib.BatchStats()
        check(lib.pc_batch_autotune(self._b, tasks, C.byref(st)))
        return {"ms": st.ms, "threads": st.threads, "ctas_per_sm": st.ctas_per_sm, "order": st.order}

    def close(self):
        if getattr(self, "_b", None):
            lib.pc_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


from . import selector  # noqa: E402
