"""The bench's multi-process path on the CPU (gloo, world size 2): the
max-over-ranks reduction and barrier used to time replicas, and a torchrun
launch of the reference arm that must print exactly one line from rank 0."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from helpers import REPO


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": "2", "LOCAL_RANK": str(rank), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    sys.path.insert(0, REPO)
    import bench
    ws, r, local, dist = bench.dist_setup()
    bench.barrier(dist)
    out[r] = bench.max_over_ranks(float(r + 1) * 1.5, dist)
    bench.barrier(dist)
    dist.destroy_process_group()


def test_max_over_ranks_and_barrier_with_two_gloo_ranks():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank_main, args=(port, out), nprocs=2, start_method="spawn", join=True)
        assert dict(out) == {0: 3.0, 1: 3.0}


def test_reference_arm_under_torchrun_prints_one_line():
    env = dict(os.environ, FVM_CPU_BUDGET_S="1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), os.path.join(REPO, "bench.py"), "--impl", "reference",
           "--workload", "euler_m3_circle", "--nx", "64", "--ny", "32", "--steps", "1", "--warmup", "3",
           "--gpus", "2"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env, cwd=REPO)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
