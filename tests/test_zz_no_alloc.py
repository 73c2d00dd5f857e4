"""The allocation-free triangle count (pc_tc_count_noalloc) against the
handle-based entry point (pc_tc), through the C ABI.

It serves callers that cannot allocate device memory (their GPU memory is
owned by another allocator or pool, or their path must not pay for an
allocation's synchronisation), so here the test plays such a caller: it
brings its own device buffers, allocated by torch before the first call, and
checks that the library allocates nothing -- the device's free memory and the
library pool's reserved bytes stay where they were across the calls.  The
largest graph (exactly 2^20 vertices, the limit) runs first and the smaller
ones after it on the same fixed scratch, each twice in a row, so counts that
read a previous call's leftovers would show.  Bad CSRs (offsets past m, a
neighbour id out of range) are turned into errors by the kernels' own bounds
checks.  This file is collected last so that a run stopping at the first
failure has run every other test."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT = 1 << 20


def _noalloc(lib, d_vl, d_el, n, m, stream):
    out = C.c_uint64()
    st = lib.pc_tc_count_noalloc(C.c_void_p(d_vl.data_ptr()), C.c_void_p(d_el.data_ptr()), n, m,
                                 C.c_void_p(stream), C.byref(out))
    return st, out.value


def _pool_reserved(device):
    """Bytes reserved by the device's default stream-ordered pool (the one
    the library's handle path allocates from), or None without cuda-python."""
    try:
        from cuda.bindings import runtime as rt
    except Exception:
        return None
    err, pool = rt.cudaDeviceGetDefaultMemPool(device)
    if err != rt.cudaError_t.cudaSuccess:
        return None
    err, v = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent)
    return int(v) if err == rt.cudaError_t.cudaSuccess else None


def test_noalloc_matches_handle_path_and_allocates_nothing(gpu, O):
    torch = pytest.importorskip("torch")
    pc = gpu
    from partitionandconquer_b200 import _lib as L
    # largest first: n = 2^20 exactly (the limit is accepted), then smaller graphs on the same scratch
    graphs = [pc.HostCSR.rmat(20, 4, 3), pc.HostCSR.rmat(14, 16, 1), pc.HostCSR.chung_lu(13, 60000, 2.1, 1024, 2),
              pc.HostCSR.er(12, 30000, 3)]
    cases = []
    for h in graphs:
        vl, el, _ = h.arrays()
        n = vl.size - 1
        g = pc.Graph(vlist=vl, elist=el)
        pg = pc.Partitioned_Graph(g, pc.equal_vertex_partition(n, 4))
        expected = pg.triangle_count()
        pg.close()
        g.close()
        assert expected == O.tc_merge(vl, el)
        cases.append((n, el.size, expected, torch.from_numpy(vl.view(np.int64)).cuda(), torch.from_numpy(el).cuda()))
    assert cases[0][0] == LIMIT
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    L.check(L.lib.pc_release_cached_memory())
    # warm-up: loads the module's kernels, which may reserve code memory once
    n, m, expected, d_vl, d_el = cases[0]
    st, got = _noalloc(L.lib, d_vl, d_el, n, m, stream)
    assert st == 0, L.lib.pc_last_error()
    assert got == expected
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    pool0 = _pool_reserved(torch.cuda.current_device())
    for n, m, expected, d_vl, d_el in cases:
        for _ in range(2):
            st, got = _noalloc(L.lib, d_vl, d_el, n, m, stream)
            assert st == 0, L.lib.pc_last_error()
            assert got == expected, (n, got, expected)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0, "device memory was allocated during allocation-free calls"
    assert _pool_reserved(torch.cuda.current_device()) == pool0


def test_noalloc_rejects_bad_csr_and_recovers(gpu):
    torch = pytest.importorskip("torch")
    pc = gpu
    from partitionandconquer_b200 import _lib as L
    vl, el, _ = pc.HostCSR.rmat(10, 8, 5).arrays()
    n, m = vl.size - 1, el.size
    want = pc.Partitioned_Graph(pc.Graph(vlist=vl, elist=el), pc.equal_vertex_partition(n, 2)).triangle_count()
    stream = torch.cuda.current_stream().cuda_stream
    d_vl = torch.from_numpy(vl.view(np.int64)).cuda()
    d_el = torch.from_numpy(el).cuda()
    # offsets ending past m: every row check runs, no row is read past the array
    bad_off = vl.copy()
    bad_off[-1] = m + 7
    st, _ = _noalloc(L.lib, torch.from_numpy(bad_off.view(np.int64)).cuda(), d_el, n, m, stream)
    assert st == 1 and b"offsets" in L.lib.pc_last_error()
    # an id >= n as the last entry of a row that is scanned as a pivot (it has
    # ids below and above itself; the row stays ascending): the kernel sees the
    # id in the row's upper part and skips it before dereferencing it
    deg = np.diff(vl).astype(np.int64)
    rows = np.repeat(np.arange(n), deg)
    dplus = np.bincount(rows[el < rows], minlength=n)
    u = int(np.flatnonzero((dplus > 0) & (dplus < deg))[0])
    bad_el = el.copy()
    bad_el[int(vl[u + 1]) - 1] = n + 100
    st, _ = _noalloc(L.lib, d_vl, torch.from_numpy(bad_el).cuda(), n, m, stream)
    assert st == 1 and b"outside" in L.lib.pc_last_error()
    # the next good call starts from a clean error word and counters
    st, got = _noalloc(L.lib, d_vl, d_el, n, m, stream)
    assert st == 0 and got == want


def test_noalloc_rejects_graphs_beyond_its_limit(gpu):
    torch = pytest.importorskip("torch")
    from partitionandconquer_b200 import _lib as L
    d = torch.zeros(16, dtype=torch.int64, device="cuda")
    st, _ = _noalloc(L.lib, d, d, LIMIT + 1, 8, 0)
    assert st == 1
    assert b"at most" in L.lib.pc_last_error()
