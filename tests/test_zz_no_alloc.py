"""The allocation-free triangle count (pc_tc_count_noalloc) against the
handle-based entry point (pc_tc), through the C ABI.

It serves callers that cannot allocate device memory, so here the test plays
such a caller: it brings its own device buffers (allocated by torch) and the
library allocates nothing.  Two calls in a row on each graph check that the
shared fixed scratch is cleared between calls.  This file is collected last
so that a run stopping at the first failure has run every other test."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib, d_vl, d_el, n, m, stream):
    out = C.c_uint64()
    st = lib.pc_tc_count_noalloc(C.c_void_p(d_vl.data_ptr()), C.c_void_p(d_el.data_ptr()), n, m,
                                 C.c_void_p(stream), C.byref(out))
    return st, out.value


def test_noalloc_matches_handle_path_twice(gpu, O):
    torch = pytest.importorskip("torch")
    pc = gpu
    from partitionandconquer_b200 import _lib as L
    graphs = [pc.HostCSR.rmat(14, 16, 1), pc.HostCSR.er(12, 30000, 3), pc.HostCSR.chung_lu(13, 60000, 2.1, 1024, 2)]
    stream = torch.cuda.current_stream().cuda_stream
    for h in graphs:
        vl, el, _ = h.arrays()
        n = vl.size - 1
        expected = pc.Partitioned_Graph(pc.Graph(vlist=vl, elist=el), pc.equal_vertex_partition(n, 4)).triangle_count()
        assert expected == O.tc_merge(vl, el)
        d_vl = torch.from_numpy(vl.view(np.int64)).cuda()
        d_el = torch.from_numpy(el).cuda()
        for _ in range(2):
            st, got = _noalloc(L.lib, d_vl, d_el, n, el.size, stream)
            assert st == 0, L.lib.pc_last_error()
            assert got == expected


def test_noalloc_rejects_graphs_beyond_its_limit(gpu):
    torch = pytest.importorskip("torch")
    from partitionandconquer_b200 import _lib as L
    d = torch.zeros(16, dtype=torch.int64, device="cuda")
    st, _ = _noalloc(L.lib, d, d, (1 << 20) + 1, 8, 0)
    assert st == 1
    assert b"at most" in L.lib.pc_last_error()
