"""Writes tests/golden/pinned_counts.json: the triangle counts of the
at-scale graphs, computed on the host cores by the CPU oracle and, where the
time allows, by the reference itself (its Graph::solve_triangle_counting_merge,
src/Graph.cpp:355-368, compiled from its own sources into oracle/_ref).

The graphs are built by the oracle's own generator (oracle/pc_graphgen.c),
which equals the product's host and device generators bit for bit; each
entry also records a fingerprint of the CSR so a GPU-side test can confirm
that it counted the same graph.

    python tests/golden/make_pinned.py [name ...]     # default: every graph

Run it in a checkout whose oracle is built (python -c 'from oracle import
oracle; oracle.build()'); it takes tens of minutes on 8 cores for the
largest graphs.  Existing entries are kept unless named on the command line.
"""
from __future__ import annotations

import json
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
OUT = Path(__file__).resolve().parent / "pinned_counts.json"

# name -> (generator, args, run the reference's own loop too)
GRAPHS = {
    "rmat16_ef16_s1": ("rmat", (16, 16, 1), True),
    "rmat20_ef16_s1": ("rmat", (20, 16, 1), True),
    "rmat22_ef16_s1": ("rmat", (22, 16, 1), True),
    "rmat24_ef16_s1": ("rmat", (24, 16, 1), True),
    "rmat25_ef16_s1": ("rmat", (25, 16, 1), False),
    "er24_m2^28_s1": ("er", (24, 1 << 28, 1), True),
    "chunglu24_m2^28_b2.1_dmax2^20_s1": ("chung_lu", (24, 1 << 28, 2.1, 1 << 20, 1), False),
}


def fingerprint(vl, el):
    """n, m, and two order-sensitive 64-bit sums of the arrays (wrapping)."""
    k = np.arange(el.size, dtype=np.uint64)
    with np.errstate(over="ignore"):
        f_el = int(np.sum(el.astype(np.uint64) * (k * np.uint64(0x9E3779B97F4A7C15) + np.uint64(1)),
                          dtype=np.uint64))
        f_vl = int(np.sum(vl.astype(np.uint64) * np.uint64(0xBF58476D1CE4E5B9), dtype=np.uint64))
    return {"n": int(vl.size - 1), "m": int(el.size), "fp_elist": f_el, "fp_vlist": f_vl}


def main(names):
    from oracle import oracle as O
    data = json.loads(OUT.read_text()) if OUT.exists() else {}
    cores = os.cpu_count() or 1
    for name in names:
        kind, args, with_ref = GRAPHS[name]
        t = time.time()
        vl, el = getattr(O, f"gen_{kind}")(*args)
        t_gen = time.time() - t
        rec = {"generator": kind, "args": list(args), **fingerprint(vl, el)}
        t = time.time()
        rec["T_oracle"] = O.tc_merge(vl, el)
        rec["oracle_s"] = round(time.time() - t, 1)
        if with_ref and O.Reference.available():
            R = O.Reference(vl, el, threads=cores)
            t = time.time()
            rec["T_reference"] = R.tc()
            rec["reference_s"] = round(time.time() - t, 1)
            R.close()
            if rec["T_reference"] != rec["T_oracle"]:
                raise SystemExit(f"{name}: reference {rec['T_reference']} != oracle {rec['T_oracle']}")
        rec["T"] = rec["T_oracle"]
        rec["host_cores"] = cores
        print(name, json.dumps(rec), f"(generated in {t_gen:.1f} s)", flush=True)
        data[name] = rec
        OUT.write_text(json.dumps(data, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    main(sys.argv[1:] or list(GRAPHS))
