"""CPU tests of the C-ABI library itself: it loads, exports every entry point
that include/pc.h declares, and its host-side code (seeded generators, the
reference's binary CSR format, input validation) behaves.  No kernel runs."""
from __future__ import annotations

import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, csr_from_edges

HEADER = ROOT / "include" / "pc.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(pc):
    from partitionandconquer_b200 import _lib
    names = declared_functions()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(_lib.lib, n)]
    assert not missing, f"declared in include/pc.h but not exported by libpc.so: {missing}"
    # and the Python binding knows every one of them
    unbound = [n for n in names if n not in _lib._SIG]
    assert not unbound, unbound


def test_version_and_device_query(pc):
    from partitionandconquer_b200 import _lib
    assert b"sm_100a" in _lib.lib.pc_version()
    assert pc.device_count() >= 0
    assert pc.launch_count() >= 0


def test_no_device_is_an_error_not_a_fallback(pc):
    if pc.device_count() > 0:
        pytest.skip("a device is present")
    vl, el = csr_from_edges(3, [(0, 1), (1, 2)])
    g = pc.Graph(vlist=vl, elist=el)
    with pytest.raises(pc.PCError) as e:
        g.solve_triangle_counting_merge()
    assert "NO_DEVICE" in str(e.value)


def test_generators_are_deterministic_and_well_formed(pc):
    a = pc.HostCSR.rmat(10, 8, 7).arrays()
    b = pc.HostCSR.rmat(10, 8, 7).arrays()
    c = pc.HostCSR.rmat(10, 8, 8).arrays()
    for x, y in zip(a[:2], b[:2]):
        np.testing.assert_array_equal(x, y)
    assert not np.array_equal(a[1], c[1])
    for h in (pc.HostCSR.rmat(11, 16, 1), pc.HostCSR.er(11, 20000, 2), pc.HostCSR.chung_lu(11, 20000, 2.1, 256, 3)):
        vl, el, _ = h.arrays()
        n = vl.size - 1
        deg = np.diff(vl).astype(np.int64)
        rows = np.repeat(np.arange(n), deg)
        # sorted, unique, no self-loops, in range
        assert np.all(el >= 0) and np.all(el < n)
        assert not np.any(rows == el)
        same_row = rows[1:] == rows[:-1]
        assert np.all(el[1:][same_row] > el[:-1][same_row])
        # symmetric
        fwd = rows.astype(np.int64) * n + el
        bwd = el.astype(np.int64) * n + rows
        np.testing.assert_array_equal(np.sort(fwd), np.sort(bwd))
        # degree-descending relabel, ties by id
        assert np.all(deg[:-1] >= deg[1:])


def test_rmat_quadrant_probabilities(pc):
    """The first recursion level picks quadrants with (0.57, 0.19, 0.19, 0.05)."""
    h = pc.HostCSR.rmat(12, 16, 3, relabel=False)
    vl, el, _ = h.arrays()
    n = vl.size - 1
    rows = np.repeat(np.arange(n), np.diff(vl).astype(np.int64))
    top_u, top_v = rows >= n // 2, el >= n // 2
    frac_low_low = np.mean(~top_u & ~top_v)
    assert 0.45 < frac_low_low < 0.7


def test_weights_symmetric_in_range(pc):
    h = pc.HostCSR.rmat(10, 8, 5).add_weights(seed=5, wmax=255)
    vl, el, w = h.arrays()
    n = vl.size - 1
    assert w.min() >= 1 and w.max() <= 255
    rows = np.repeat(np.arange(n), np.diff(vl).astype(np.int64))
    key_f = rows.astype(np.int64) * n + el
    key_b = el.astype(np.int64) * n + rows
    of, ob = np.argsort(key_f), np.argsort(key_b)
    np.testing.assert_array_equal(w[of], w[ob])


def test_binfile_round_trip(pc, tmp_path):
    h = pc.HostCSR.rmat(9, 8, 2).add_weights(seed=2, wmax=100)
    h.save(str(tmp_path))
    for f in ("csr_vlist.bin", "csr_elist.bin", "csr_weight.bin"):
        assert (tmp_path / f).exists()
    # the reference's layout: uint64 offsets, int32 ids and weights
    vl0, el0, w0 = h.arrays()
    np.testing.assert_array_equal(np.fromfile(tmp_path / "csr_vlist.bin", np.uint64), vl0)
    np.testing.assert_array_equal(np.fromfile(tmp_path / "csr_elist.bin", np.int32), el0)
    g = pc.Graph(str(tmp_path), True)
    np.testing.assert_array_equal(g.get_csr_vlist(), vl0)
    np.testing.assert_array_equal(g.get_csr_elist(), el0)
    np.testing.assert_array_equal(g.get_csr_weight(), w0)
    assert g.get_vertex_num() == vl0.size - 1 and g.get_edge_num() == el0.size


@pytest.mark.parametrize("bad", ["nonmonotone", "out_of_range", "wrong_total", "truncated_file"])
def test_host_validation_rejects_malformed_csr(pc, tmp_path, bad):
    vl, el = csr_from_edges(4, [(0, 1), (1, 2), (2, 3)])
    if bad == "nonmonotone":
        vl = vl.copy(); vl[2] = 1; vl[1] = 3
    elif bad == "out_of_range":
        el = el.copy(); el[0] = 9
    elif bad == "wrong_total":
        vl = vl.copy(); vl[-1] += 1
    if bad == "truncated_file":
        vl.tofile(tmp_path / "csr_vlist.bin")
        (tmp_path / "csr_elist.bin").write_bytes(el.tobytes()[:-2])
        with pytest.raises(pc.PCError) as e:
            pc.HostCSR.load(str(tmp_path))
    else:
        with pytest.raises(pc.PCError) as e:
            pc.HostCSR.from_arrays(vl, el)
    assert "INVALID_INPUT" in str(e.value)


def test_missing_csr_dir_is_an_error(pc, tmp_path):
    with pytest.raises(pc.PCError):
        pc.HostCSR.load(str(tmp_path / "nope"))


def test_equal_vertex_partition(pc):
    v = pc.equal_vertex_partition(65536, 64)
    assert v.dtype == np.int32 and v.min() == 0 and v.max() == 63
    assert np.all(np.bincount(v) == 1024)
    assert np.all(np.diff(v) >= 0)


def test_result_buffers_are_validated_on_the_host(pc):
    """Every result method takes an optional caller-owned `out`; a buffer of
    the wrong size, dtype, layout or writability is refused before any
    device work, and a good one is used as is."""
    from partitionandconquer_b200 import _result
    got = _result(None, 5, np.int32)
    assert got.dtype == np.int32 and got.size == 5
    buf = np.zeros(7, np.float32)
    assert _result(buf, 7, np.float32) is buf
    for bad in (np.zeros(6, np.float32),              # size
                np.zeros(7, np.float64),              # dtype
                np.zeros(14, np.float32)[::2],        # not contiguous
                [0.0] * 7):                           # not an array
        with pytest.raises(ValueError):
            _result(bad, 7, np.float32)
    ro = np.zeros(7, np.float32)
    ro.flags.writeable = False
    with pytest.raises(ValueError):
        _result(ro, 7, np.float32)
