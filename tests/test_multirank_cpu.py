"""The multi-rank (torchrun) plumbing of bench.py on CPU: two gloo ranks on
127.0.0.1. Timing is the max over ranks; the reference arm runs on rank 0
alone and prints one JSON line, the other ranks exit 0 without work."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
torch = pytest.importorskip("torch")


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


RANK_SCRIPT = r"""
import datetime, json, os, sys
sys.path.insert(0, %r)
import torch, torch.distributed as dist
import bench
world, rank, local = bench.dist_setup(None)
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
v = bench.reduce_max(torch, dist, 1.5 + rank)
dist.barrier()
print(json.dumps({"rank": rank, "world": world, "max": v}))
dist.destroy_process_group()
"""


def run_ranks(args_for_rank, env_extra=None, timeout=120):
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        env.update(env_extra or {})
        procs.append(subprocess.Popen(args_for_rank(rank), cwd=ROOT, env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            out, err = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        outs.append((p.returncode, out, err))
    return outs


def test_two_gloo_ranks_take_the_max_over_ranks():
    outs = run_ranks(lambda rank: [sys.executable, "-c", RANK_SCRIPT % ROOT])
    for rc, out, err in outs:
        assert rc == 0, err
    got = [json.loads(out.strip().splitlines()[-1]) for _, out, _ in outs]
    assert sorted(g["rank"] for g in got) == [0, 1]
    assert all(g["world"] == 2 and g["max"] == 2.5 for g in got)


def test_reference_arm_prints_once_on_rank_zero():
    cmd = [sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--workload", "config1",
           "--steps", "1", "--warmup", "0"]
    outs = run_ranks(lambda rank: cmd, timeout=600)
    (rc0, out0, err0), (rc1, out1, err1) = outs
    assert rc0 == 0, err0[-2000:]
    assert rc1 == 0, err1[-2000:]
    lines0 = [l for l in out0.splitlines() if l.startswith("{")]
    assert len(lines0) == 1
    line = json.loads(lines0[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert not [l for l in out1.splitlines() if l.startswith("{")]
