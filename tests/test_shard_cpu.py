"""Dec-band sharding on the host: the band plan, and the assembly of band
slabs on rank 0 over two gloo ranks (127.0.0.1). The bands' gridding itself
runs on the GPU (tests/test_gpu_shard.py)."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from hcgrid_b200 import shard

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("ny,parts", [(1200, 1), (1200, 2), (1200, 8), (48, 3), (40, 4), (7, 2), (100, 7)])
def test_plan_covers_rows_with_aligned_edges(ny, parts):
    b = shard.plan(ny, parts)
    assert len(b) == parts
    assert b[0][0] == 0 and b[-1][1] == ny
    for (a0, a1), (c0, c1) in zip(b, b[1:]):
        assert a1 == c0  # contiguous
    for y0, y1 in b:
        assert y0 <= y1
        assert y0 % shard.ALIGN == 0 and (y1 % shard.ALIGN == 0 or y1 == ny)
    sizes = [(y1 - y0 + shard.ALIGN - 1) // shard.ALIGN for y0, y1 in b]
    assert max(sizes) - min(sizes) <= 1


def test_plan_rejects_no_parts():
    with pytest.raises(ValueError):
        shard.plan(10, 0)


def test_assemble_single_rank_is_identity():
    c = np.arange(12, dtype=np.float32).reshape(6, 2)
    w = np.ones(6, np.float32)
    got_c, got_w = shard.assemble(None, 0, 1, [(0, 3)], 2, c, w)
    assert got_c is c and got_w is w


RANK_SCRIPT = r"""
import datetime, json, sys
sys.path.insert(0, %r)
import numpy as np
import torch.distributed as dist
from hcgrid_b200 import shard
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
rank, world = dist.get_rank(), dist.get_world_size()
nx, ny, nchan = 5, 40, 3
bands = shard.plan(ny, world)
y0, y1 = bands[rank]
rows = np.arange(y0 * nx, y1 * nx)
cube = (rows[:, None] * 10 + np.arange(nchan)[None, :]).astype(np.float32)
w = rows.astype(np.float32) + 0.5
c, ww = shard.assemble(dist, rank, world, bands, nx, cube, w)
if rank == 0:
    want = np.arange(ny * nx)
    ok = np.array_equal(c, (want[:, None] * 10 + np.arange(nchan)[None, :]).astype(np.float32)) and \
        np.array_equal(ww, want.astype(np.float32) + 0.5)
    print(json.dumps({"rank": 0, "ok": bool(ok), "bands": bands}))
else:
    print(json.dumps({"rank": rank, "none": c is None and ww is None}))
dist.destroy_process_group()
"""


def test_assemble_over_two_gloo_ranks():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_SCRIPT % ROOT], cwd=ROOT, env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            out, err = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    assert outs[0]["ok"] and outs[0]["bands"] == [[0, 16], [16, 40]]
    assert outs[1]["none"]
