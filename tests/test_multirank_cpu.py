"""Multi-rank logic of bench.py on CPU (gloo, world size 2).

bench.py runs one process per GPU under torchrun; every rank steps its own
replica, the timed region is bracketed by a barrier, the reported time is the
max over ranks, and only rank 0 prints.  These tests exercise that logic with
the gloo backend on 127.0.0.1, without a GPU.
"""

import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": "2",
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(ROOT))
    import bench
    ws, r, local = bench.dist_env()
    dist = bench.init_dist(ws, "gloo")
    bench.barrier(dist)
    worst = bench.max_over_ranks(dist, 1.5 + r)
    bench.barrier(dist)
    scene, meta = bench.make_workload("cube", r)
    dist.destroy_process_group()
    out.put((r, ws, worst, float(scene.positions[0, 0]), meta["particles"]))


def test_max_over_ranks_and_barrier_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort()
    assert [g[0] for g in got] == [0, 1]
    assert all(g[1] == 2 for g in got)
    assert all(g[2] == 2.5 for g in got)          # max over ranks seen by every rank
    assert got[0][3] != got[1][3]                 # each rank steps its own replica (own seed)
    assert got[0][4] == got[1][4]                 # of the same size: weak scaling


def test_reference_arm_prints_once_under_torchrun():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--reference-budget-s", "1"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
