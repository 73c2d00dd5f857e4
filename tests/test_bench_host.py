"""Host-side pieces of bench.py: the algorithmic byte counts of a triangle
count, the CSR fingerprint that finds a graph's pinned count, and the oracle
parity check (a planted mismatch in the oracle's role fails the run)."""
from __future__ import annotations

import itertools

import numpy as np
import pytest

import bench


def _brute(vl, el):
    n = vl.size - 1
    N = [set(el[vl[u]:vl[u + 1]].tolist()) for u in range(n)]
    dplus = np.array([sum(1 for v in N[u] if v < u) for u in range(n)], np.int64)
    W = sum(int(dplus[u] + dplus[v]) for u in range(n) for v in N[u] if v < u)
    # pivot form: for every oriented edge c -> b (b < c), the ids of N(c) below b
    scan = sum(sum(1 for a in N[c] if a < b) for c in range(n) for b in N[c] if b < c)
    tri = sum(1 for a, b, c in itertools.combinations(range(n), 3) if b in N[a] and c in N[a] and c in N[b])
    return dplus, W, scan, tri


def test_tc_bytes_match_brute_force(O):
    vl, el = O.gen_rmat(7, 8, 3)
    dplus, W, scan, tri = _brute(vl, el)
    tb = bench.tc_bytes(vl, el, chunk_rows=17)
    n, m = vl.size - 1, el.size
    assert tb["e_plus"] == int(dplus.sum()) == m // 2
    assert tb["W"] == W
    assert tb["wedges"] == scan
    assert tb["pivot_bytes"] == 8 * (n + 1) + 4 * m + 4 * n + 12 * (m // 2) + 4 * scan
    assert tb["merge_bytes"] == 4 * W + 12 * (m // 2) + 8 * (n + 1)
    assert O.tc_merge(vl, el) == tri


def test_pinned_lookup_by_fingerprint(O):
    vl, el = O.gen_rmat(16, 16, 1)
    assert bench.pinned_count(vl, el) == ("rmat16_ef16_s1", 15643386)
    el2 = el.copy()
    el2[[0, 1]] = el2[[1, 0]]
    assert bench.pinned_count(vl, el2) == (None, None)


def test_tc_parity_fails_on_mismatch(O):
    vl, el = O.gen_rmat(10, 8, 1)
    T = O.tc_merge(vl, el)
    rec = bench.tc_parity(O, vl, el, T, 1)
    assert rec["match"] and rec["oracle_T"] == T
    with pytest.raises(SystemExit):
        bench.tc_parity(O, vl, el, T + 1, 1)


def test_jaccard_parity_full_and_audited(O):
    vl, el = O.gen_rmat(10, 16, 2)
    J = O.jaccard_edges(vl, el)
    T = O.tc_merge(vl, el)
    assert bench.jaccard_parity(O, vl, el, J, T)["jaccard_match"]
    audited = bench.jaccard_parity(O, vl, el, J, T, full_limit=0, sample_rows=50)
    assert audited["jaccard_match"] and audited["jaccard_sum_counts"] == 6 * T
    bad = J.copy()
    bad[np.flatnonzero(J > 0)[3]] += np.float32(0.25)
    assert not bench.jaccard_parity(O, vl, el, bad, T, full_limit=0, sample_rows=50)["jaccard_match"]
