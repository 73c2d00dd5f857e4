"""The host-side drop-in pieces: the `pc_main preprocess` task reproduces the
reference's preprocess tool byte for byte (text loader, CSR files, log2-range
weights), and the CLI's argument handling.  CPU only; the algorithm tasks of
the CLI are covered by the gpu tests."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

from conftest import ROOT

PC_MAIN = ROOT / "partitionandconquer_b200" / "bin" / "pc_main"
REF_PRE = ROOT / "oracle" / "_ref" / "preprocess"


def write_edge_list(path, rng, n, m, one_based):
    lines = ["# comment line", "% another comment"]
    for _ in range(m):
        u, v = rng.integers(0, n, 2)
        if one_based:
            u, v = u + 1, v + 1
        lines.append(f"{u} {v}")
    lines.append(f"{3 + one_based} {3 + one_based}")  # a self-loop, dropped
    lines.append(lines[3])  # a duplicate edge
    path.write_text("\n".join(lines) + "\n")


@pytest.mark.parametrize("one_based", [0, 1])
def test_preprocess_matches_reference(tmp_path, one_based):
    if not PC_MAIN.exists():
        pytest.skip("pc_main not built")
    if not REF_PRE.exists():
        pytest.skip("reference preprocess tool not built in this checkout (oracle/_ref)")
    rng = np.random.default_rng(10 + one_based)
    for tool, d in ((str(PC_MAIN), tmp_path / "ours"), (str(REF_PRE), tmp_path / "ref")):
        (d / "origin").mkdir(parents=True)
        write_edge_list(d / "graph.txt", np.random.default_rng(10 + one_based), 300, 2000, one_based)
        args = [tool, "preprocess", str(d) + "/", "graph.txt"] if tool == str(PC_MAIN) else [tool, str(d) + "/", "graph.txt"]
        r = subprocess.run(args, capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr
    for f in ("csr_vlist.bin", "csr_elist.bin", "csr_weight.bin"):
        a = (tmp_path / "ours" / "origin" / f).read_bytes()
        b = (tmp_path / "ref" / "origin" / f).read_bytes()
        assert a == b, f
    w = np.fromfile(tmp_path / "ours" / "origin" / "csr_weight.bin", np.int32)
    assert w.min() >= 1 and w.max() <= int(np.log2(300))


def test_cli_rejects_bad_usage():
    if not PC_MAIN.exists():
        pytest.skip("pc_main not built")
    r = subprocess.run([str(PC_MAIN)], capture_output=True, text=True)
    assert r.returncode == 2
    r = subprocess.run([str(PC_MAIN), "tc", "/nonexistent"], capture_output=True, text=True)
    assert r.returncode == 2
    r = subprocess.run([str(PC_MAIN), "nope"], capture_output=True, text=True)
    assert r.returncode == 2
