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


TENSOR_SCRIPT = r"""
import datetime, json, sys
sys.path.insert(0, %r)
import numpy as np
import torch
import torch.distributed as dist
from hcgrid_b200 import shard
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
rank, world = dist.get_rank(), dist.get_world_size()
nx, ny, nchan = 5, 40, 3
bands = shard.plan(ny, world)
y0, y1 = bands[rank]
rows = torch.arange(y0 * nx, y1 * nx, dtype=torch.float32)
cube = rows[:, None] * 10 + torch.arange(nchan, dtype=torch.float32)[None, :]
c, ww = shard.assemble_tensors(dist, rank, world, bands, nx, cube, rows + 0.5)
if rank == 0:
    want = torch.arange(ny * nx, dtype=torch.float32)
    ok = torch.equal(c, want[:, None] * 10 + torch.arange(nchan, dtype=torch.float32)[None, :]) and \
        torch.equal(ww, want + 0.5)
    print(json.dumps({"rank": 0, "ok": bool(ok)}))
else:
    print(json.dumps({"rank": rank, "none": c is None and ww is None}))
dist.destroy_process_group()
"""


def _run_ranks(script, world=2):
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", script % ROOT], cwd=ROOT, env=env,
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
    return outs


def test_assemble_tensors_gathers_unequal_bands_over_gloo():
    """The tensor gather behind the band-sharded bench (NCCL on CUDA tensors
    there): unequal bands (16 and 24 rows) padded to equal sizes, unpadded
    into the whole cube on rank 0."""
    outs = _run_ranks(TENSOR_SCRIPT)
    assert outs[0]["ok"] and outs[1]["none"]


# The band sample range, argued in hcgrid_b200/csrc/hcg_shard.cu, checked with
# the FP64 oracle on the CPU: complete rings of the band, one sample in front.

def _band_range(g, ps, xw, yw, p0, p1):
    """hcg_field_band_samples' rule from the oracle's per-pixel ring ranges."""
    from oracle import oracle as O
    lo, hi = None, None
    for p in range(p0, p1):
        ur, dr, _, _, _ = O.pixel_windows(g, ps, xw[p], yw[p])
        if dr >= ur:
            lo = ur if lo is None else min(lo, ur)
            hi = dr if hi is None else max(hi, dr)
    if lo is None:
        return 0, 0
    rlo, rend = lo - ps.firstring, hi - ps.firstring + 1
    a, b = int(ps.lut[rlo]), int(ps.lut[rend])
    if b <= a:
        return 0, 0
    return (a - 1 if a > 0 else 0), b


@pytest.mark.parametrize("case", ["synth_dec40", "synth_polar", "synth_wrap"])
def test_band_sample_ranges_grid_bands_exactly(case):
    from conftest import load_case
    from oracle import oracle as O
    c = load_case(case)
    g = O.prepare_grid_kernel(float(c["sigma"]), float(c["sphere_radius"]), float(c["hpx_max_res"]))
    lon, lat = c["lon"], c["lat"]
    vals = np.asarray(c["values"], np.float64).reshape(len(lon), -1)[:, 0]
    ps = O.presort(g.hpx, lon, lat)
    xw, yw = c["xwcs"], c["ywcs"]
    nx, ny = int(c["nx"]), int(c["ny"])
    whole, ww, _ = O.grid(g, ps, lon[ps.perm], lat[ps.perm], vals[ps.perm], xw, yw)
    for y0, y1 in shard.plan(ny, 3):
        p0, p1 = y0 * nx, y1 * nx
        s0, s1 = _band_range(g, ps, xw, yw, p0, p1)
        if s1 == s0:
            assert np.all(ww[p0:p1] == 0)
            continue
        assert s1 - s0 < len(lon)  # a part of the samples
        idx = ps.perm[s0:s1]
        gb = O.prepare_grid_kernel(float(c["sigma"]), float(c["sphere_radius"]), float(c["hpx_max_res"]))
        pb = O.presort(gb.hpx, lon[idx], lat[idx])
        cb, wb, _ = O.grid(gb, pb, lon[idx][pb.perm], lat[idx][pb.perm], vals[idx][pb.perm], xw[p0:p1], yw[p0:p1])
        np.testing.assert_array_equal(wb, ww[p0:p1])
        np.testing.assert_array_equal(cb, whole[p0:p1])

