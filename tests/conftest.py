"""Shared fixtures.  Tests marked `gpu` need a CUDA device and call libpc.so
through its C ABI; everything else runs on the CPU (oracle, host code, ABI
symbol table, multi-process logic over gloo)."""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"
GOLDEN_GRAPHS = ["tiny", "k6", "star", "path", "isolated", "rmat10", "er10"]
INT_MAX = 2**31 - 1


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs libpc.so kernels")


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def golden_summary() -> dict:
    return json.loads((GOLDEN / "rmat16_summary.json").read_text())


@pytest.fixture(scope="session")
def pc():
    import partitionandconquer_b200 as m
    return m


@pytest.fixture(scope="session")
def O():
    from oracle import oracle as m
    m.clib()
    return m


@pytest.fixture(scope="session")
def gpu(pc):
    """Skips nothing: a gpu-marked test on a machine without a device fails loudly."""
    if pc.device_count() < 1:
        pytest.fail("no CUDA device visible: gpu tests need a B200")
    return pc


def csr_from_edges(n, edges):
    adj = [set() for _ in range(n)]
    for u, v in edges:
        if u != v:
            adj[u].add(v)
            adj[v].add(u)
    vl = np.zeros(n + 1, np.uint64)
    el = []
    for u in range(n):
        row = sorted(adj[u])
        el.extend(row)
        vl[u + 1] = vl[u] + len(row)
    return vl, np.asarray(el, np.int32)


def small_graphs(pc):
    """Hand graphs plus seeded random ones, as (name, vlist, elist, weights)."""
    out = []
    for name in GOLDEN_GRAPHS:
        d = load_golden(name)
        out.append((name, d["vlist"], d["elist"], d["weights"]))
    for seed in (1, 2):
        h = pc.HostCSR.rmat(11, 8, seed).add_weights(seed, 255)
        out.append((f"rmat11s{seed}", *h.arrays()))
    h = pc.HostCSR.er(11, 16384, 9).add_weights(9, 255)
    out.append(("er11", *h.arrays()))
    h = pc.HostCSR.chung_lu(11, 16384, 2.1, 512, 4).add_weights(4, 255)
    out.append(("cl11", *h.arrays()))
    h = pc.HostCSR.rmat(10, 16, 6, relabel=False).add_weights(6, 255)
    out.append(("rmat10_raw_ids", *h.arrays()))
    return out
