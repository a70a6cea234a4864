"""Replicas across ranks (the path does not shard): the bench's cross-rank
logic -- max-over-ranks timing, whole-job rate, rank-0-only reference arm --
on two gloo ranks on the CPU."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


WORKER = r"""
import os, sys, json
sys.path.insert(0, {root!r})
import torch.distributed as dist
import bench
rank, world, local = bench.dist_env()
dist.init_process_group("gloo", init_method="env://")
ms = 2.0 + rank            # rank 1 is the slower replica
m = bench.max_over_ranks(ms, dist, "cpu")
rate = bench.whole_job_rate(world, 1000, m)
dist.barrier()
print(json.dumps({{"rank": rank, "max_ms": m, "rate": rate}}))
dist.destroy_process_group()
"""


def test_two_gloo_ranks_take_the_max_time():
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER.format(root=ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=120) for p in procs]
    import json
    res = [json.loads(o[0].strip().splitlines()[-1]) for o in outs]
    for r in res:
        assert r["max_ms"] == 3.0
        assert abs(r["rate"] - 2 * 1000 / 3e-3 / 1e6) < 1e-9


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
