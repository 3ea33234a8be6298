"""The N > 1 path of bench.py on CPU: two gloo ranks, no GPU.

bench.py shards at request level (one replica per GPU, no collective on the
data path); torch.distributed supplies only the barrier and the max-over-ranks
timing. These tests run bench.py's own plumbing (dist_setup, barrier,
max_over_ranks, dist_teardown) in two processes over gloo, and check that the
reference arm does its work on rank 0 alone."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys, json
sys.path.insert(0, {root!r})
import bench
rank, world, local = bench.dist_setup()
assert world == 2 and rank in (0, 1)
bench.barrier(world)
import torch
mx = bench.max_over_ranks(10.0 + rank, world, torch.device("cpu"))
bench.dist_teardown(world)
print(json.dumps({{"rank": rank, "max": mx}}))
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _launch(code, env_extra, timeout=120):
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="", **env_extra)
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            out, err = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        assert p.returncode == 0, err[-2000:]
        outs.append(out)
    return outs


def test_gloo_barrier_and_max_over_ranks():
    import json
    outs = _launch(WORKER.format(root=ROOT), {})
    got = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert sorted(g["rank"] for g in got) == [0, 1]
    assert all(g["max"] == 11.0 for g in got)  # every rank sees the slowest rank's time


def test_reference_arm_runs_on_rank_zero_only():
    """bench.run_reference returns None on every rank but 0 (no work, exit 0)."""
    code = f"""
import sys
sys.path.insert(0, {ROOT!r})
import bench
class A: steps = 1
print(bench.run_reference(A(), 1, 2))
"""
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "None"
