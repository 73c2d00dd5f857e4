"""Benchmark: triangle counting (the intersection hot path) on RMAT scale 24,
edge factor 16, seed 1, degree-relabelled, 1024 equal-vertex partitions.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one Partitioned_Graph::solve_triangle_counting_merge over the whole
graph.  Rank 0 prints one JSON line.

 * value   -- GTEPS = undirected edges / device time of one step, graph
              resident in HBM (CUDA events on the library's stream), with the
              learned per-partition selector (PC_VARIANT_AUTO).
 * e2e     -- the same through the C ABI from pinned host buffers: CSR upload
              (validated), partition view, plan, counting, 8-byte result read.
 * roofline -- SURVEY's algorithmic bytes of triangle counting,
              B = 4 W + 12 |E+| + 8 (n+1) with W = sum over oriented edges of
              (d+(u) + d+(v)), over the summed duration of the counting
              kernels, against the measured HBM copy bandwidth.
 * cpu_baseline -- the reference's own loop (Graph::solve_triangle_counting_merge,
              src/Graph.cpp:358-365, calling Graph::cnt_common_neis_less_than_merge)
              over an every-k-th-row sample on all host cores, extrapolated.
With N > 1 (torchrun) every rank runs an independent replica on its own GPU
(the path does not shard: replicas only); value = all ranks' edges / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "intersection GTEPS on RMAT-24 ef16; % HBM roofline; learned vs plain selector"
PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--partitions", type=int, default=1024)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-sample-seconds", type=float, default=8.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--train-scale", type=int, default=22)
    ap.add_argument("--profile", action="store_true",
                    help="profiling run: plain heuristic plan only, no selector training, e2e or CPU leg")
    return ap.parse_args()


# ---- distributed plumbing (replicas) ------------------------------------------

class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
            self.backend = backend
            self.dist = dist
            self.torch = torch

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if self.world == 1:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64,
                              device="cuda" if self.backend == "nccl" else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.barrier()
            self.dist.destroy_process_group()


# ---- workload -------------------------------------------------------------------

def make_graph(pc, scale, ef, seed):
    t = time.time()
    h = pc.HostCSR.rmat(scale, ef, seed)
    vl, el, _ = h.arrays()
    return vl, el, time.time() - t


def tc_algorithmic_bytes(vl, el, chunk_rows=1 << 20):
    """B_TC = 4 W + 12 |E+| + 8 (n+1), W = sum over oriented edges (u -> v, v < u)
    of d+(u) + d+(v) with d+(x) = |N(x) & [0, x)| (the merge read volume).
    Computed in row chunks to bound host memory."""
    n = vl.size - 1
    deg = np.diff(vl).astype(np.int64)
    dplus = np.zeros(n, np.int64)
    for lo in range(0, n, chunk_rows):
        hi = min(n, lo + chunk_rows)
        rows = np.repeat(np.arange(lo, hi, dtype=np.int64), deg[lo:hi])
        seg = el[vl[lo]:vl[hi]]
        dplus[lo:hi] = np.bincount(rows[seg < rows] - lo, minlength=hi - lo)
    W = int((dplus * dplus).sum())
    for lo in range(0, n, chunk_rows):
        hi = min(n, lo + chunk_rows)
        rows = np.repeat(np.arange(lo, hi, dtype=np.int64), deg[lo:hi])
        seg = el[vl[lo]:vl[hi]]
        W += int(dplus[seg[seg < rows]].sum())
    e_plus = int(dplus.sum())
    return 4 * W + 12 * e_plus + 8 * (n + 1), W, e_plus


def hbm_peak():
    try:
        p = json.loads(PEAKS.read_text())
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi samples every 200 ms during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for name, val in zip(names, f[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---- the reference arm ----------------------------------------------------------

def reference_tc_sample(vl, el, target_s, threads):
    """Times the reference's TC loop on every k-th row; returns (GTEPS, sample)."""
    from oracle import oracle as O
    n = vl.size - 1
    e_plus = el.size // 2
    if O.Reference.available():
        R = O.Reference(vl, el, threads=threads)
        run = R.tc_rows
        kind = "reference"
    else:
        R = None
        run = lambda rows: O.tc_rows(vl, el, rows)  # noqa: E731
        kind = "port"
    k = 4096
    while True:
        rows = np.arange(0, n, k, dtype=np.int32)
        t = time.perf_counter()
        run(rows)
        dt = time.perf_counter() - t
        if dt * 4 >= target_s or k == 1:
            break
        k = max(1, int(k * max(dt, 1e-3) / target_s * 1.5)) if dt > 0.05 else max(1, k // 16)
    gteps = e_plus / (dt * k) / 1e9
    sample = (f"rows u = 0 mod {k} ({rows.size} of {n} rows) of the RMAT-24 graph, "
              f"{dt:.2f} s, extrapolated x{k}")
    return gteps, kind, sample, R, run, rows, k, e_plus


def run_reference_arm(args, dist):
    import partitionandconquer_b200 as pc
    vl, el, _ = make_graph(pc, args.scale, args.edge_factor, args.seed)
    threads = os.cpu_count() or 1
    gteps, kind, sample, R, run, rows, k, e_plus = reference_tc_sample(vl, el, args.cpu_sample_seconds, threads)
    for _ in range(args.warmup):
        run(rows)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        run(rows)
        times.append(time.perf_counter() - t)
    step_s = statistics.median(times) * k
    value = e_plus / step_s / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": "GTEPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step_s * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded RMAT)",
        "config": {"workload": f"tc_rmat{args.scale}_ef{args.edge_factor}", "partitions": args.partitions,
                   "path": "Graph::solve_triangle_counting_merge loop (the partitioned constructor needs P*n "
                           "offsets plus 2*P*n vectors: infeasible in memory at this size)"},
        "cpu_baseline": {"value": round(value, 6), "unit": "GTEPS", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": round(value, 6), "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if R is not None:
        R.close()


# ---- our arm ------------------------------------------------------------------------

def train_selector(pc, args):
    """Training data generated by the method itself on separate graphs (RMAT
    seed 2 at the training scale, ER and Chung-Lu): per-unit timings of every
    variant; then the MLP is trained on the GPU and the heuristic autotuned on
    the same samples."""
    sel = pc.selector
    sel.clear()
    s = args.train_scale
    graphs = [pc.HostCSR.rmat(s, args.edge_factor, args.seed + 1),
              pc.HostCSR.er(s - 2, 1 << (s + 2), args.seed + 2),
              pc.HostCSR.chung_lu(s - 2, 1 << (s + 2), 2.1, 1 << (s - 6), args.seed + 3)]
    for h in graphs:
        vl, el, _ = h.arrays()
        n = vl.size - 1
        g = pc.Graph(vlist=vl, elist=el)
        pg = pc.Partitioned_Graph(g, pc.equal_vertex_partition(n, max(1, n // 16384)))
        sel.collect(pg, max_units=96, repeats=2)
        pg.close()
        g.close()
    tuned = sel.autotune()
    loss = sel.train(steps=1500, lr=3e-3, seed=7)
    return {"samples": sel.num_samples(), "train_loss": loss, "heuristic_params": tuned.tolist()}


def time_device(pc, torch, pg, stream, variant, steps, warmup):
    for _ in range(warmup):
        pg.triangle_count(variant=variant)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    times, kms, counts = [], [], set()
    launches0 = pc.launch_count()
    for _ in range(steps):
        ev[0].record(stream)
        c, st = pg.triangle_count(variant=variant, stats=True)
        ev[1].record(stream)
        ev[1].synchronize()
        times.append(ev[0].elapsed_time(ev[1]))
        kms.append(st.kernel_ms)
        counts.add(c)
    launches = pc.launch_count() - launches0
    return times, kms, counts, launches, st


def run_ours(args, dist):
    import torch

    import partitionandconquer_b200 as pc
    dev = dist.local if dist.world > 1 else 0
    torch.cuda.set_device(dev)
    from partitionandconquer_b200 import _lib
    _lib.check(_lib.lib.pc_set_device(dev))
    if dist.world > 1:
        os.environ.setdefault("OMP_NUM_THREADS", str(max(1, (os.cpu_count() or 1) // dist.world)))
    vl, el, t_gen = make_graph(pc, args.scale, args.edge_factor, args.seed)
    n = vl.size - 1
    algo_bytes, W, e_plus = tc_algorithmic_bytes(vl, el)
    v2p = pc.equal_vertex_partition(n, args.partitions)
    if args.profile:
        g = pc.Graph(vlist=vl, elist=el)
        pg = pc.Partitioned_Graph(g, v2p)
        stream = torch.cuda.ExternalStream(g.stream())
        t, k, c, launches, st = time_device(pc, torch, pg, stream, pc.VARIANT_HEURISTIC, args.steps, args.warmup)
        print(json.dumps({"profile": True, "workload": f"tc_rmat{args.scale}_ef{args.edge_factor}_p{args.partitions}",
                          "ms": statistics.median(t), "kernel_ms": statistics.median(k), "triangles": c.pop(),
                          "launches_per_step": launches / max(1, args.steps),
                          "variants_per_unit": list(st.variant_hist)}), flush=True)
        pg.close()
        g.close()
        return
    train = train_selector(pc, args)

    g = pc.Graph(vlist=vl, elist=el)
    pg = pc.Partitioned_Graph(g, v2p)
    stream = torch.cuda.ExternalStream(g.stream())

    # learned (headline) and plain heuristic, interleaved to share clock conditions
    dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clocks:
        t_learned, k_learned, c_learned, launches, st_learned = time_device(pc, torch, pg, stream, pc.VARIANT_AUTO,
                                                                            args.steps, args.warmup)
        t_plain, k_plain, c_plain, _, st_plain = time_device(pc, torch, pg, stream, pc.VARIANT_HEURISTIC,
                                                             args.steps, args.warmup)
    torch.cuda.synchronize()
    dist.barrier()
    if len(c_learned | c_plain) != 1:
        raise SystemExit(f"inconsistent triangle counts: {c_learned | c_plain}")
    T = c_learned.pop()
    step_ms = statistics.median(t_learned)
    step_ms_max = dist.max(step_ms)
    plain_ms = statistics.median(t_plain)
    value = dist.world * e_plus / (step_ms_max / 1e3) / 1e9

    # roofline of the counting kernels (event-timed inside the call on the same stream)
    kernel_ms = statistics.median(k_learned)
    peak, peak_kind = hbm_peak()
    achieved = algo_bytes / (kernel_ms / 1e3) / 1e9
    traffic = None
    tf = ROOT / "profiles" / "tc_rmat24_traffic.txt"
    if tf.exists():
        for ln in tf.read_text().splitlines():
            if ln.startswith("dram_bytes_per_call="):
                traffic = float(ln.split("=", 1)[1])

    # end to end through the C ABI from pinned host buffers
    from partitionandconquer_b200 import _lib as L
    pinned = []
    for a in (vl, el, v2p):
        L.check(L.lib.pc_host_register(L.ptr(a), a.nbytes))
        pinned.append(a)
    e2e = []
    for i in range(args.e2e_steps + 1):
        t = time.perf_counter()
        g2 = pc.Graph(vlist=vl, elist=el)
        pg2 = pc.Partitioned_Graph(g2, v2p)
        c = pg2.triangle_count(variant=pc.VARIANT_AUTO)
        pg2.close()
        g2.close()
        dt = time.perf_counter() - t
        if c != T:
            raise SystemExit("e2e count mismatch")
        if i > 0:
            e2e.append(dt)
    for a in pinned:
        L.lib.pc_host_unregister(L.ptr(a))
    e2e_s = dist.max(statistics.median(e2e))
    e2e_value = dist.world * e_plus / e2e_s / 1e9
    h2d = vl.nbytes + el.nbytes + v2p.nbytes

    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        gteps, kind, sample, R, *_ = reference_tc_sample(vl, el, args.cpu_sample_seconds, os.cpu_count() or 1)
        cpu = {"value": round(gteps, 6), "unit": "GTEPS", "cores": os.cpu_count() or 1, "kind": kind,
               "sample": sample}
        if R is not None:
            R.close()

    if dist.rank == 0:
        hist = list(st_learned.variant_hist)
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": "GTEPS", "n_gpus": dist.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step_ms_max, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded RMAT, generated in-process)",
            "config": {
                "workload": f"tc_rmat{args.scale}_ef{args.edge_factor}_p{args.partitions}",
                "graph": f"RMAT(0.57,0.19,0.19,0.05) scale {args.scale} ef {args.edge_factor} seed {args.seed}, "
                         "symmetrised, deduplicated, degree-relabelled", "n": int(n), "m_directed": int(el.size),
                "undirected_edges": int(e_plus), "partitions": args.partitions, "triangles": int(T),
                "l2": "inputs larger than L2 (CSR %.2f GB)" % ((vl.nbytes + el.nbytes) / 1e9),
                "selector": "learned (MLP judged by the autotuned heuristic)",
                "parallelism": "replicas" if dist.world > 1 else "1 GPU",
                "plan_variants_per_unit": hist,
            },
            "learned_vs_plain": {"learned_ms": round(step_ms, 4), "plain_ms": round(plain_ms, 4),
                                 "speedup": round(plain_ms / step_ms, 4),
                                 "plain_variants_per_unit": list(st_plain.variant_hist), **train},
            "e2e": {"value": round(e2e_value, 4), "unit": "GTEPS", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": 8, "ms_per_step": round(e2e_s * 1e3, 2)},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic, "peak_kind": peak_kind,
                         "algorithmic_bytes": int(algo_bytes), "W": int(W), "kernel_ms": round(kernel_ms, 4)},
            "cpu_baseline": cpu,
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
            "setup": {"graph_gen_s": round(t_gen, 2)},
        }
        print(json.dumps(line), flush=True)
    pg.close()
    g.close()


def main():
    args = parse()
    if args.impl == "reference":
        # the reference is a host-CPU program: rank 0 alone runs it, no process group
        if int(os.environ.get("RANK", "0")) == 0:
            run_reference_arm(args, None)
        return
    dist = Dist()
    try:
        run_ours(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
