"""Serving loop (hcg_server): continuous batching over two lanes with
footprint admission; every served cube equals the single-call cube."""
import numpy as np
import pytest

from hcgrid_b200 import api

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from test_gpu_batch import SHAPES, make  # noqa: E402


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def test_served_jobs_equal_single_calls(ctx):
    jobs = [make(ctx, s) for s in SHAPES]
    ctx.synchronize()
    srv = api.Server(ctx, lanes=2, hbm_budget=1 << 30, max_batch=3)
    try:
        outs, tickets = [], []
        for rep in range(3):
            for job, f, t in jobs:
                P = t.nx * t.ny
                cube = torch.full((P * job.nchan,), float("inf"), device="cuda")
                w = torch.full((P,), float("inf"), device="cuda")
                tickets.append(srv.submit(f, t, cube, w, footprint=4 * P * (job.nchan + 1)))
                outs.append((job, f, t, cube, w))
        lat = [srv.wait(tk) for tk in tickets]
        srv.drain()
        st = srv.stats()
    finally:
        srv.close()
    assert st["jobs"] == len(tickets) and st["batches"] >= 2
    assert all(l[0] > 0 for l in lat) and st["p99_s"] >= st["p50_s"] > 0
    for job, f, t, cube, w in outs:
        ref_cube, ref_w = ctx.grid(f, t)
        np.testing.assert_array_equal(cube.cpu().numpy(), ref_cube.reshape(-1))
        np.testing.assert_array_equal(w.cpu().numpy(), ref_w)


def test_served_tensor_core_jobs_equal_single_calls(ctx):
    """Multi-channel fields with split spectra run on the persistent
    tensor-core kernel inside the lanes' batches; each served cube equals
    the field's single hcg_grid cube, while jobs overlap on the device."""
    jobs = [make(ctx, s) for s in SHAPES]
    for job, f, t in jobs:
        if job.nchan > 1:
            f.split_spectra(api.ENGINE_TC_F16, keep_fp32=False)
    ctx.synchronize()
    srv = api.Server(ctx, lanes=2, hbm_budget=1 << 30, max_batch=2)
    try:
        outs, tickets = [], []
        for rep in range(2):
            for job, f, t in jobs:
                P = t.nx * t.ny
                cube = torch.full((P * job.nchan,), float("inf"), device="cuda")
                w = torch.full((P,), float("inf"), device="cuda")
                tickets.append(srv.submit(f, t, cube, w, footprint=4 * P * (job.nchan + 1)))
                outs.append((job, f, t, cube, w))
        for tk in tickets:
            srv.wait(tk)
        st = srv.stats()
    finally:
        srv.close()
    assert st["jobs"] == len(tickets)
    for job, f, t, cube, w in outs:
        ref_cube, ref_w = ctx.grid(f, t)
        np.testing.assert_array_equal(cube.cpu().numpy(), ref_cube.reshape(-1))
        np.testing.assert_array_equal(w.cpu().numpy(), ref_w)
