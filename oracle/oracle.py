"""TEST INFRASTRUCTURE -- numpy wrappers over the CPU oracle.

``C``   : liboracle.so, the plain-C restatement (pc_oracle.c).
``REF`` : _ref/libpcref.so, the reference's own Graph.cpp with a C entry layer
          (ref_capi.cpp), present when it was built (see Makefile).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libpcref.so"
# the reference checkout: PC_REFERENCE_DIR, else `reference` beside the repository
REF_SRC = Path(os.environ.get("PC_REFERENCE_DIR", str(HERE.parent.parent / "reference")))

P = C.c_void_p
i32, u64, f32, f64 = C.c_int32, C.c_uint64, C.c_float, C.c_double


def build(ref: bool = True):
    """Builds liboracle.so, and the reference library when its sources exist."""
    subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True)
    if ref and (REF_SRC / "src" / "Graph.cpp").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={REF_SRC}"], check=True)


def _ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


class _Mute:
    """Sends the process's stdout (fd 1) to /dev/null while the reference's
    own printf progress lines run, so callers keep a clean stdout."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        C.CDLL(None).fflush(None)
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *a):
        C.CDLL(None).fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def _load_c():
    if not ORACLE_SO.exists():
        build(ref=False)
    lib = C.CDLL(str(ORACLE_SO))
    sig = {
        "or_tc_merge": (u64, [u64, P, P]),
        "or_tc_galloping": (u64, [u64, P, P]),
        "or_tc_rows": (u64, [u64, P, P, P, u64]),
        "or_layout": (C.c_int, [u64, P, P, P, P, i32, P, P, P]),
        "or_tc_partitioned": (u64, [u64, P, P, i32]),
        "or_lcc": (None, [u64, P, P, P]),
        "or_jaccard_edges": (None, [u64, P, P, P]),
        "or_jaccard_queries": (None, [u64, P, P, P, i32, P]),
        "or_jaccard_rows": (None, [u64, P, P, P, u64, P]),
        "or_jaccard_audit": (None, [u64, P, P, P, P, P, P]),
        "or_batch_pairs": (None, [u64, P, P, P, u64, P]),
        "or_batch_sets": (None, [u64, P, P, P, P, u64, P]),
        "or_bfs": (None, [u64, P, P, i32, P]),
        "or_sssp": (None, [u64, P, P, P, i32, P]),
        "or_pagerank_f64": (None, [u64, P, P, f64, i32, P, P]),
        "or_kcore": (i32, [u64, P, P, P]),
        "or_mis": (None, [u64, P, P, P]),
        "or_mis_priority": (None, [u64, P, P, P, P]),
        "or_cdlp": (None, [u64, P, P, i32, P]),
        "or_friend_triangle": (u64, [u64, P, P, i32, P, u64]),
        "or_square_count": (u64, [u64, P, P]),
        "og_rmat": (P, [C.c_uint32, u64, u64, C.c_int]),
        "og_er": (P, [C.c_uint32, u64, u64, C.c_int]),
        "og_chung_lu": (P, [C.c_uint32, u64, f64, u64, u64, C.c_int]),
        "og_rmat_batch": (P, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, u64, P]),
        "og_n": (u64, [P]),
        "og_m": (u64, [P]),
        "og_copy": (None, [P, P, P]),
        "og_free": (None, [P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_C = None


def clib():
    global _C
    if _C is None:
        _C = _load_c()
    return _C


def _csr(vl, el):
    vl = np.ascontiguousarray(vl, np.uint64)
    el = np.ascontiguousarray(el, np.int32)
    return vl, el, vl.size - 1


# ---- seeded graphs (pc_graphgen.c) -------------------------------------------------

def _take(h):
    if not h:
        raise MemoryError("graph generation failed")
    lib = clib()
    n, m = int(lib.og_n(h)), int(lib.og_m(h))
    vl = np.empty(n + 1, np.uint64)
    el = np.empty(m, np.int32)
    lib.og_copy(h, _ptr(vl), _ptr(el))
    lib.og_free(h)
    return vl, el


def gen_rmat(scale, edge_factor, seed, relabel=True):
    """RMAT(0.57, 0.19, 0.19, 0.05) with 2^scale vertices and 2^scale *
    edge_factor draws, symmetrised, deduplicated, degree-relabelled."""
    return _take(clib().og_rmat(scale, edge_factor, seed, int(relabel)))


def gen_er(scale, nedges, seed, relabel=True):
    return _take(clib().og_er(scale, nedges, seed, int(relabel)))


def gen_chung_lu(scale, nedges, beta, dmax, seed, relabel=True):
    return _take(clib().og_chung_lu(scale, nedges, beta, dmax, seed, int(relabel)))


def gen_rmat_batch(G, smin, smax, emin, emax, seed=0):
    voff = np.empty(G + 1, np.uint64)
    vl, el = _take(clib().og_rmat_batch(G, smin, smax, emin, emax, seed, _ptr(voff)))
    return vl, el, voff


# ---- the C restatement ---------------------------------------------------------

def tc_merge(vl, el):
    vl, el, n = _csr(vl, el)
    return int(clib().or_tc_merge(n, _ptr(vl), _ptr(el)))


def friend_triangle(vl, el, root, nodes):
    vl, el, n = _csr(vl, el)
    q = np.ascontiguousarray(nodes, np.int32)
    return int(clib().or_friend_triangle(n, _ptr(vl), _ptr(el), int(root), _ptr(q), q.size))


def square_count(vl, el):
    vl, el, n = _csr(vl, el)
    return int(clib().or_square_count(n, _ptr(vl), _ptr(el)))


def tc_rows(vl, el, rows):
    vl, el, n = _csr(vl, el)
    r = np.ascontiguousarray(rows, np.int32)
    return int(clib().or_tc_rows(n, _ptr(vl), _ptr(el), _ptr(r), r.size))


def tc_galloping(vl, el):
    vl, el, n = _csr(vl, el)
    return int(clib().or_tc_galloping(n, _ptr(vl), _ptr(el)))


def layout(vl, el, w, v2p):
    vl, el, n = _csr(vl, el)
    v2p = np.ascontiguousarray(v2p, np.int32)
    P_ = int(v2p.max()) + 1 if n else 1
    ovl = np.empty(P_ * n + 1, np.uint64)
    oel = np.empty(el.size, np.int32)
    ow = None if w is None else np.empty(el.size, np.int32)
    wa = None if w is None else np.ascontiguousarray(w, np.int32)
    clib().or_layout(n, _ptr(vl), _ptr(el), _ptr(wa), _ptr(v2p), P_, _ptr(ovl), _ptr(oel), _ptr(ow))
    return ovl, oel, ow


def tc_partitioned(pvl, pel, n, P_):
    pvl = np.ascontiguousarray(pvl, np.uint64)
    pel = np.ascontiguousarray(pel, np.int32)
    return int(clib().or_tc_partitioned(n, _ptr(pvl), _ptr(pel), P_))


def lcc(vl, el):
    vl, el, n = _csr(vl, el)
    out = np.empty(n, np.float64)
    clib().or_lcc(n, _ptr(vl), _ptr(el), _ptr(out))
    return out


def jaccard_edges(vl, el):
    vl, el, n = _csr(vl, el)
    out = np.empty(el.size, np.float32)
    clib().or_jaccard_edges(n, _ptr(vl), _ptr(el), _ptr(out))
    return out


def jaccard_rows(vl, el, rows):
    """Exact all-edge Jaccard values of the listed rows, concatenated."""
    vl, el, n = _csr(vl, el)
    r = np.ascontiguousarray(rows, np.int32)
    d = (vl[r.astype(np.int64) + 1] - vl[r.astype(np.int64)]).astype(np.int64)
    out = np.empty(int(d.sum()), np.float32)
    clib().or_jaccard_rows(n, _ptr(vl), _ptr(el), _ptr(r), r.size, _ptr(out))
    return out


def jaccard_audit(vl, el, J):
    """(sum of recovered common-neighbour counts (= 6 T), entries that do not
    round-trip, entries whose twin differs) for an all-edge Jaccard result."""
    vl, el, n = _csr(vl, el)
    J = np.ascontiguousarray(J, np.float32)
    if J.size != el.size:
        raise ValueError("one Jaccard value per CSR entry expected")
    res = [C.c_uint64() for _ in range(3)]
    clib().or_jaccard_audit(n, _ptr(vl), _ptr(el), _ptr(J), *(C.byref(x) for x in res))
    return tuple(int(x.value) for x in res)


def jaccard_queries(vl, el, q):
    vl, el, n = _csr(vl, el)
    q = np.ascontiguousarray(q, np.int32)
    out = np.empty(q.size * q.size, np.float64)
    clib().or_jaccard_queries(n, _ptr(vl), _ptr(el), _ptr(q), q.size, _ptr(out))
    return out


def batch_pairs(vl, el, pairs):
    vl, el, n = _csr(vl, el)
    pairs = np.ascontiguousarray(pairs, np.int32).reshape(-1)
    out = np.empty(pairs.size // 2, np.uint64)
    clib().or_batch_pairs(n, _ptr(vl), _ptr(el), _ptr(pairs), pairs.size // 2, _ptr(out))
    return out


def batch_sets(vl, el, sets):
    vl, el, n = _csr(vl, el)
    ids = np.concatenate([np.asarray(s, np.int32) for s in sets]) if sets else np.zeros(0, np.int32)
    offs = np.zeros(len(sets) + 1, np.uint64)
    np.cumsum([len(s) for s in sets], out=offs[1:])
    out = np.empty(len(sets), np.uint64)
    clib().or_batch_sets(n, _ptr(vl), _ptr(el), _ptr(ids), _ptr(offs), len(sets), _ptr(out))
    return out


def bfs(vl, el, src):
    vl, el, n = _csr(vl, el)
    out = np.empty(n, np.int32)
    clib().or_bfs(n, _ptr(vl), _ptr(el), src, _ptr(out))
    return out


def sssp(vl, el, w, src):
    vl, el, n = _csr(vl, el)
    w = np.ascontiguousarray(w, np.int32)
    out = np.empty(n, np.int32)
    clib().or_sssp(n, _ptr(vl), _ptr(el), _ptr(w), src, _ptr(out))
    return out


def pagerank_f64(vl, el, damping=0.85, iters=20, init=None):
    vl, el, n = _csr(vl, el)
    out = np.empty(n, np.float64)
    ini = None if init is None else np.ascontiguousarray(init, np.float64)
    clib().or_pagerank_f64(n, _ptr(vl), _ptr(el), damping, iters, _ptr(ini), _ptr(out))
    return out


def kcore(vl, el):
    vl, el, n = _csr(vl, el)
    out = np.empty(n, np.int32)
    largest = clib().or_kcore(n, _ptr(vl), _ptr(el), _ptr(out))
    return out, int(largest)


def mis(vl, el, priority=None):
    vl, el, n = _csr(vl, el)
    out = np.zeros(n, np.int32)
    if priority is None:
        clib().or_mis(n, _ptr(vl), _ptr(el), _ptr(out))
    else:
        pr = np.ascontiguousarray(priority, np.uint64)
        clib().or_mis_priority(n, _ptr(vl), _ptr(el), _ptr(pr), _ptr(out))
    return out


def cdlp(vl, el, labels, iters=10):
    vl, el, n = _csr(vl, el)
    lab = np.ascontiguousarray(labels, np.int32).copy()
    clib().or_cdlp(n, _ptr(vl), _ptr(el), iters, _ptr(lab))
    return lab


# ---- the reference itself (oracle/_ref) ------------------------------------------

def _muted(fn):
    def wrap(*a, **k):
        with _Mute():
            return fn(*a, **k)
    wrap.__name__ = fn.__name__
    wrap.__doc__ = fn.__doc__
    return wrap


class Reference:
    """The reference library (libpcref.so) on one graph, written to a temporary
    CSR directory in the reference's binary format and loaded by its own
    Graph(csrdir, is_weighted) constructor."""

    _lib = None

    @classmethod
    def available(cls) -> bool:
        return REF_SO.exists()

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not REF_SO.exists():
                raise FileNotFoundError(f"{REF_SO} not built")
            lib = C.CDLL(str(REF_SO))
            sig = {
                "ref_graph_load": (P, [C.c_char_p, C.c_int]),
                "ref_graph_free": (None, [P]),
                "ref_graph_n": (u64, [P]),
                "ref_graph_m": (u64, [P]),
                "ref_pgraph_new": (P, [P, P, u64, C.c_int]),
                "ref_pgraph_free": (None, [P]),
                "ref_pgraph_partitions": (u64, [P]),
                "ref_pgraph_reorder": (None, [P]),
                "ref_pgraph_layout": (None, [P, P, P, P]),
                "ref_pgraph_evaluate": (None, [P]),
                "ref_tc_graph": (u64, [P, C.c_int, C.c_int]),
                "ref_tc_pgraph": (u64, [P, C.c_int]),
                "ref_tc_rows": (u64, [P, P, u64, C.c_int]),
                "ref_lcc_graph": (None, [P, C.c_int, C.c_int, P]),
                "ref_lcc_pgraph": (None, [P, C.c_int, P]),
                "ref_jsim_graph": (None, [P, P, i32, C.c_int, P]),
                "ref_jsim_pgraph": (None, [P, P, i32, P]),
                "ref_batch_pairs": (None, [P, C.c_int, P, u64, C.c_int, P]),
                "ref_batch_sets": (None, [P, C.c_int, P, P, u64, C.c_int, P]),
                "ref_bfs_graph": (None, [P, i32, P]),
                "ref_sssp": (None, [P, C.c_int, u64, i32, P]),
                "ref_pagerank": (None, [P, C.c_int, u64, f32, C.c_int, C.c_int, P]),
                "ref_kcore": (None, [P, C.c_int, u64, C.c_int, P]),
                "ref_mis": (None, [P, C.c_int, u64, C.c_int, P]),
                "ref_cdlp": (None, [P, C.c_int, u64, C.c_int, C.c_int, P]),
                "ref_friend_triangle": (u64, [P, C.c_int, C.c_int, i32, P, u64, C.c_int]),
                "ref_square_count": (u64, [P]),
            }
            for name, (res, args) in sig.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            cls._lib = lib
        return cls._lib

    def __init__(self, vl, el, w=None, v2p=None, threads=None, csrdir=None):
        lib = self.lib()
        self.threads = threads or os.cpu_count() or 1
        self._tmp = None
        if csrdir is None:
            self._tmp = tempfile.TemporaryDirectory(prefix="pcref_")
            csrdir = self._tmp.name
            np.ascontiguousarray(vl, np.uint64).tofile(os.path.join(csrdir, "csr_vlist.bin"))
            np.ascontiguousarray(el, np.int32).tofile(os.path.join(csrdir, "csr_elist.bin"))
            if w is not None:
                np.ascontiguousarray(w, np.int32).tofile(os.path.join(csrdir, "csr_weight.bin"))
        with _Mute():
            self.g = lib.ref_graph_load(csrdir.encode(), int(w is not None))
        self.n = int(lib.ref_graph_n(self.g))
        self.m = int(lib.ref_graph_m(self.g))
        self.pg = None
        if v2p is not None:
            self.v2p = np.ascontiguousarray(v2p, np.int32)
            with _Mute():
                self.pg = lib.ref_pgraph_new(self.g, _ptr(self.v2p), self.n, self.threads)

    def close(self):
        lib = self.lib()
        if self.pg:
            lib.ref_pgraph_free(self.pg)
            self.pg = None
        if self.g:
            lib.ref_graph_free(self.g)
            self.g = None
        if self._tmp is not None:
            self._tmp.cleanup()
            self._tmp = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _obj(self, partitioned):
        if partitioned and not self.pg:
            raise ValueError("no partition given")
        return self.pg if partitioned else self.g

    @_muted
    def tc(self, partitioned=False, galloping=False):
        lib = self.lib()
        if partitioned:
            return int(lib.ref_tc_pgraph(self.pg, int(galloping)))
        return int(lib.ref_tc_graph(self.g, int(galloping), self.threads))

    @_muted
    def tc_rows(self, rows):
        r = np.ascontiguousarray(rows, np.int32)
        return int(self.lib().ref_tc_rows(self.g, _ptr(r), r.size, self.threads))

    @_muted
    def layout(self):
        P_ = int(self.lib().ref_pgraph_partitions(self.pg))
        vl = np.empty(P_ * self.n + 1, np.uint64)
        el = np.empty(self.m, np.int32)
        self.lib().ref_pgraph_layout(self.pg, _ptr(vl), _ptr(el), None)
        return vl, el

    @_muted
    def reorder(self):
        self.lib().ref_pgraph_reorder(self.pg)

    @_muted
    def lcc(self, partitioned=False, galloping=False):
        out = np.empty(self.n, np.float64)
        if partitioned:
            self.lib().ref_lcc_pgraph(self.pg, int(galloping), _ptr(out))
        else:
            self.lib().ref_lcc_graph(self.g, int(galloping), self.threads, _ptr(out))
        return out

    @_muted
    def jsim(self, q, partitioned=False):
        q = np.ascontiguousarray(q, np.int32)
        out = np.empty(q.size * q.size, np.float64)
        if partitioned:
            self.lib().ref_jsim_pgraph(self.pg, _ptr(q), q.size, _ptr(out))
        else:
            self.lib().ref_jsim_graph(self.g, _ptr(q), q.size, self.threads, _ptr(out))
        return out

    @_muted
    def batch_pairs(self, pairs, partitioned=False):
        p = np.ascontiguousarray(pairs, np.int32).reshape(-1)
        out = np.empty(p.size // 2, np.uint64)
        self.lib().ref_batch_pairs(self._obj(partitioned), int(partitioned), _ptr(p), p.size // 2, self.threads,
                                   _ptr(out))
        return out

    @_muted
    def batch_sets(self, sets, partitioned=False):
        ids = np.concatenate([np.asarray(s, np.int32) for s in sets])
        offs = np.zeros(len(sets) + 1, np.uint64)
        np.cumsum([len(s) for s in sets], out=offs[1:])
        out = np.empty(len(sets), np.uint64)
        self.lib().ref_batch_sets(self._obj(partitioned), int(partitioned), _ptr(ids), _ptr(offs), len(sets),
                                  self.threads, _ptr(out))
        return out

    @_muted
    def bfs_parents(self, src):
        out = np.empty(self.n, np.int32)
        self.lib().ref_bfs_graph(self.g, src, _ptr(out))
        return out

    @_muted
    def sssp(self, src, partitioned=False):
        out = np.empty(self.n, np.int32)
        self.lib().ref_sssp(self._obj(partitioned), int(partitioned), self.n, src, _ptr(out))
        return out

    @_muted
    def pagerank(self, damping=0.85, iters=20, partitioned=True):
        out = np.empty(self.n, np.float32)
        self.lib().ref_pagerank(self._obj(partitioned), int(partitioned), self.n, damping, iters, self.threads,
                                _ptr(out))
        return out

    @_muted
    def kcore(self, partitioned=False):
        out = np.empty(self.n, np.int32)
        self.lib().ref_kcore(self._obj(partitioned), int(partitioned), self.n, self.threads, _ptr(out))
        return out

    @_muted
    def mis(self, partitioned=False):
        out = np.empty(self.n, np.int32)
        self.lib().ref_mis(self._obj(partitioned), int(partitioned), self.n, self.threads, _ptr(out))
        return out

    @_muted
    def friend_triangle(self, root, nodes, partitioned=False, galloping=False):
        q = np.ascontiguousarray(nodes, np.int32)
        return int(self.lib().ref_friend_triangle(self._obj(partitioned), int(partitioned), int(galloping), root,
                                                  _ptr(q), q.size, self.threads))

    @_muted
    def square_count(self):
        return int(self.lib().ref_square_count(self._obj(True)))

    @_muted
    def cdlp(self, labels, iters=10, partitioned=False):
        lab = np.ascontiguousarray(labels, np.int32).copy()
        self.lib().ref_cdlp(self._obj(partitioned), int(partitioned), self.n, iters, self.threads, _ptr(lab))
        return lab
