"""bench.py's multi-GPU mode runs independent replicas (the path does not
shard); its only collective plumbing is a barrier and a max over ranks of the
step time.  Exercised here with two gloo ranks on the CPU."""
from __future__ import annotations

import os
import socket
import sys

import pytest

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(ROOT))
    import bench
    d = bench.Dist()
    assert d.backend == "gloo"
    d.barrier()
    m = d.max(float(rank + 1) * 1.5)
    d.close()
    q.put((rank, m))


def test_replica_max_over_ranks_gloo():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("the gloo path is the CPU one")
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert res == [(0, 3.0), (1, 3.0)]


def test_reference_arm_runs_on_rank0_only(tmp_path):
    """Under torchrun the reference arm runs on rank 0 alone; other ranks exit
    at once without touching a process group."""
    import subprocess
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--scale", "10"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
