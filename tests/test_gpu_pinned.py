"""Full-size triangle counts against the pinned values.

tests/golden/pinned_counts.json holds the counts of the at-scale graphs,
computed on the host cores by the oracle and -- for RMAT-16 to RMAT-24 -- by
the reference's own Graph::solve_triangle_counting_merge (src/Graph.cpp:355-368)
compiled from its sources (tests/golden/make_pinned.py).  Here the graph is
generated and built on the GPU, its CSR fingerprint must equal the pinned
graph's, and the learned and plain plans must both return the pinned count:
the metric graph (RMAT-24, 1024 partitions) and config 2's RMAT-22 (256
partitions) at full size."""
from __future__ import annotations

import json

import pytest

import bench
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,P", [("rmat22_ef16_s1", 256), ("rmat24_ef16_s1", 1024)])
def test_full_size_count_equals_pinned(gpu, name, P):
    pc = gpu
    rec = json.loads((GOLDEN / "pinned_counts.json").read_text())[name]
    scale, ef, seed = rec["args"]
    g = pc.Graph.rmat_device(scale, ef, seed)
    vl, el = g.get_csr_vlist(), g.get_csr_elist()
    fp = bench.csr_fingerprint(vl, el)
    assert all(fp[k] == rec[k] for k in fp), (fp, rec)
    del vl, el
    pg = pc.Partitioned_Graph(g, pc.equal_vertex_partition(rec["n"], P))
    assert pg.triangle_count(variant=pc.VARIANT_AUTO) == rec["T"]
    assert pg.triangle_count(variant=pc.VARIANT_HEURISTIC) == rec["T"]
    pg.close()
    g.close()
