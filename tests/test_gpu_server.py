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


def test_large_jobs_run_alone_and_errors_do_not_stall_the_server(ctx):
    """A job whose target has at least 2^20 pixels runs alone on a lane
    (hcg_grid path, on a lane context that was never prepared) beside batches
    of small jobs; its cube equals the single call's. A failing job reports
    its error, and closing the server with jobs still queued returns once
    they are done."""
    big = dict(block=9, n=40_000, size_deg=1.0, ra=80.0, dec=10.0, grid=1024, nchan=4, fwhm=180.0, seed=29)
    jobs = [make(ctx, s) for s in [big] + SHAPES]
    ctx.synchronize()
    bad_field = ctx.field(jobs[1][0].lon, jobs[1][0].lat)  # no spectra
    srv = api.Server(ctx, lanes=2, hbm_budget=1 << 32, max_batch=4)
    try:
        outs, tickets = [], []
        for job, f, t in jobs:
            P = t.nx * t.ny
            cube = torch.full((P * job.nchan,), float("inf"), device="cuda")
            w = torch.full((P,), float("inf"), device="cuda")
            tickets.append(srv.submit(f, t, cube, w, footprint=4 * P * (job.nchan + 1)))
            outs.append((job, f, t, cube, w))
        for tk in tickets:
            srv.wait(tk)
        P1 = jobs[1][2].nx * jobs[1][2].ny
        bad = srv.submit(bad_field, jobs[1][2], torch.empty(P1, device="cuda"), None, footprint=4 * P1)
        with pytest.raises(RuntimeError):
            srv.wait(bad)
        # queued work at close: the lanes finish it before the server goes
        for job, f, t in jobs[1:]:
            P = t.nx * t.ny
            srv.submit(f, t, torch.empty(P * job.nchan, device="cuda"), None, footprint=4 * P)
    finally:
        srv.close()
    bad_field.close()
    for job, f, t, cube, w in outs:
        ref_cube, ref_w = ctx.grid(f, t)
        np.testing.assert_array_equal(cube.cpu().numpy(), ref_cube.reshape(-1))
        np.testing.assert_array_equal(w.cpu().numpy(), ref_w)
