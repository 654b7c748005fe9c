"""Batch engine (hcg_grid_batch): persistent work-queue launches replayed
from one CUDA graph. Each job's cube must equal what hcg_grid writes for
the job on its own (same device arithmetic, same summation order), whether
it runs alone or inside a mixed batch, and match the oracle."""
import numpy as np
import pytest

from hcgrid_b200 import api, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


SHAPES = [
    dict(block=0, n=30_000, size_deg=0.8, ra=40.0, dec=20.0, grid=48, nchan=1, fwhm=180.0, seed=21),
    dict(block=1, n=60_000, size_deg=1.0, ra=120.0, dec=60.0, grid=64, nchan=64, fwhm=300.0, seed=22),
    dict(block=2, n=25_000, size_deg=0.5, ra=200.0, dec=-20.0, grid=40, nchan=96, fwhm=60.0, seed=23),
    dict(block=3, n=40_000, size_deg=1.2, ra=310.0, dec=75.0, grid=56, nchan=256, fwhm=180.0, seed=24),
    dict(block=4, n=20_000, size_deg=0.6, ra=10.0, dec=-5.0, grid=32, nchan=1, fwhm=300.0, seed=25),
]


def make(ctx, shape):
    job = synth.block_job(shape)
    kp = np.array([job.sigma_deg, 0.0, 0.0])
    ctx.prepare_grid_kernel(api.GAUSS1D, kp, job.sphere_radius, job.hpx_max_res)
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(np.ascontiguousarray(job.values.reshape(job.n, -1)))
    f.nchan = job.nchan
    t = ctx.target_from_header(job.header)
    return job, f, t


@pytest.fixture(scope="module")
def jobs(ctx):
    return [make(ctx, s) for s in SHAPES]


def run_batch(ctx, items, layouts):
    outs = []
    spec = []
    for (job, f, t), lay in zip(items, layouts):
        P = t.nx * t.ny
        cube = torch.full((P * job.nchan,), float("inf"), dtype=torch.float32, device="cuda")
        w = torch.full((P,), float("inf"), dtype=torch.float32, device="cuda")
        outs.append((cube, w))
        spec.append((f, t, cube, w, lay))
    ctx.grid_batch(spec)
    torch.cuda.synchronize()
    return [(c.cpu().numpy(), w.cpu().numpy()) for c, w in outs]


def single(ctx, job, f, t, layout):
    cube, w = ctx.grid(f, t, layout=layout)
    return cube.reshape(-1), w


def test_batch_equals_single_calls(ctx, jobs):
    layouts = [api.SAMPLE_MAJOR, api.CHANNEL_MAJOR, api.SAMPLE_MAJOR, api.CHANNEL_MAJOR, api.SAMPLE_MAJOR]
    got = run_batch(ctx, jobs, layouts)
    for (job, f, t), lay, (cube, w) in zip(jobs, layouts, got):
        ref_cube, ref_w = single(ctx, job, f, t, lay)
        np.testing.assert_array_equal(cube, ref_cube)
        np.testing.assert_array_equal(w, ref_w)


def test_job_alone_equals_job_in_mix(ctx, jobs):
    mix = run_batch(ctx, jobs, [api.SAMPLE_MAJOR] * len(jobs))
    for i in (1, 3):
        alone = run_batch(ctx, [jobs[i]], [api.SAMPLE_MAJOR])[0]
        np.testing.assert_array_equal(alone[0], mix[i][0])
        np.testing.assert_array_equal(alone[1], mix[i][1])


def test_batch_replay_after_growth(ctx, jobs):
    """A larger batch after a small one (pool and scratch grow, the captured
    graph is replayed unchanged)."""
    small = run_batch(ctx, jobs[:1], [api.SAMPLE_MAJOR])
    big = run_batch(ctx, jobs + jobs, [api.SAMPLE_MAJOR] * (2 * len(jobs)))
    np.testing.assert_array_equal(small[0][0], big[0][0])
    for i in range(len(jobs)):
        np.testing.assert_array_equal(big[i][0], big[i + len(jobs)][0])


def test_batch_past_the_job_table_capacity(ctx, jobs):
    """A batch of more jobs than the job table holds (64 at first) after a
    small one: the table is reallocated and the captured graphs, which take
    its address, are captured again; every cube equals the single call's."""
    run_batch(ctx, jobs[:2], [api.SAMPLE_MAJOR] * 2)
    many = (jobs * 15)[:70]
    got = run_batch(ctx, many, [api.SAMPLE_MAJOR] * len(many))
    ref = [single(ctx, job, f, t, api.SAMPLE_MAJOR) for job, f, t in jobs]
    for i, (cube, w) in enumerate(got):
        np.testing.assert_array_equal(cube, ref[i % len(jobs)][0])
        np.testing.assert_array_equal(w, ref[i % len(jobs)][1])
    again = run_batch(ctx, jobs[:2], [api.SAMPLE_MAJOR] * 2)  # and a small batch after it
    np.testing.assert_array_equal(again[1][0], ref[1][0])


def test_batch_jobs_match_oracle(ctx, jobs):
    got = run_batch(ctx, jobs, [api.SAMPLE_MAJOR] * len(jobs))
    for (job, f, t), (cube, w) in zip(jobs, got):
        xw, yw = t.coords()
        g = O.prepare_grid_kernel(job.sigma_deg, job.sphere_radius, job.hpx_max_res)
        ps = O.presort(g.hpx, job.lon, job.lat)
        vals = job.values.reshape(job.n, -1).astype(np.float64)
        oc, ow, _ = O.grid(g, ps, job.lon[ps.perm], job.lat[ps.perm], vals[ps.perm], xw, yw)
        ref = oc / ow[:, None]
        c = cube.reshape(-1, job.nchan)
        nan = np.isnan(ref)
        assert np.array_equal(np.isnan(c), nan)
        tol = 1e-6 if job.nchan == 1 else 1e-5
        for ch in range(job.nchan):
            r = ref[~nan[:, ch], ch]
            if r.size:
                assert np.abs(c[~nan[:, ch], ch] - r).max() / np.abs(r).max() <= tol


@pytest.fixture(scope="module")
def tc_jobs(ctx):
    """Fresh fields of the same shapes; the multi-channel ones hold split
    spectra (FP16 hi/lo for blocks 1 and 3, BF16 hi/lo for block 2), so the
    batch runs them on the persistent tensor-core kernel."""
    items = [make(ctx, s) for s in SHAPES]
    for i, eng in ((1, api.ENGINE_TC_F16), (2, api.ENGINE_TC_BF16), (3, api.ENGINE_TC_F16)):
        items[i][1].split_spectra(eng)
    return items


def test_tensor_core_batch_equals_single_calls(ctx, tc_jobs, jobs):
    layouts = [api.CHANNEL_MAJOR, api.SAMPLE_MAJOR, api.CHANNEL_MAJOR, api.SAMPLE_MAJOR, api.CHANNEL_MAJOR]
    got = run_batch(ctx, tc_jobs, layouts)
    st = ctx.stats()
    assert st.tc_macs > 0
    for i, ((job, f, t), lay, (cube, w)) in enumerate(zip(tc_jobs, layouts, got)):
        ref_cube, ref_w = single(ctx, job, f, t, lay)  # hcg_grid, engine of the field's split
        np.testing.assert_array_equal(cube, ref_cube)
        np.testing.assert_array_equal(w, ref_w)
        # and within the split's precision of the FP32 engine
        j32, f32, t32 = jobs[i]
        c32, w32 = single(ctx, j32, f32, t32, lay)
        np.testing.assert_array_equal(w, w32)
        if job.nchan > 1:
            nan = np.isnan(c32)
            np.testing.assert_array_equal(np.isnan(cube), nan)
            scale = np.abs(c32[~nan]).max()
            assert np.abs(cube[~nan] - c32[~nan]).max() <= 5e-5 * scale


@pytest.mark.parametrize("shape", range(api.BATCH_SHAPES))
def test_tensor_core_batch_shapes_equal_single_calls(ctx, tc_jobs, shape):
    """Every pipeline shape of the batch pass's tensor-core kernel (channels
    per item, slots per chunk, stages) gives the single call's cube bit for
    bit."""
    ctx.batch_set_shape(shape)
    try:
        got = run_batch(ctx, tc_jobs, [api.SAMPLE_MAJOR] * len(tc_jobs))
    finally:
        ctx.batch_set_shape(-1)
    for (job, f, t), (cube, w) in zip(tc_jobs, got):
        ref_cube, ref_w = single(ctx, job, f, t, api.SAMPLE_MAJOR)
        np.testing.assert_array_equal(cube, ref_cube)
        np.testing.assert_array_equal(w, ref_w)


def test_batch_autotuner_picks_a_shape_per_channel_class(ctx, tc_jobs):
    """hcg_autotune_batch times every shape per channel class of the batch's
    tensor-core jobs (64 channels: class 0, 96: class 1, 256: class 2), keeps
    the fastest, and the tuned batch still equals the single calls."""
    spec = []
    for job, f, t in tc_jobs:
        P = t.nx * t.ny
        spec.append((f, t, torch.empty((P * job.nchan,), device="cuda"), torch.empty((P,), device="cuda"),
                     api.SAMPLE_MAJOR))
    try:
        res = ctx.autotune_batch(spec, reps=2)
        assert sorted(r["channel_class"] for r in res) == [0, 1, 2]
        for r in res:
            assert r["jobs"] == 1 and 0 <= r["shape"] < api.BATCH_SHAPES
            assert all(m > 0 for m in r["ms"]) and r["ms"][r["shape"]] == min(r["ms"]) and r["spread"] >= 0
        got = run_batch(ctx, tc_jobs, [api.SAMPLE_MAJOR] * len(tc_jobs))
    finally:
        ctx.batch_set_shape(-1)
    for (job, f, t), (cube, w) in zip(tc_jobs, got):
        ref_cube, ref_w = single(ctx, job, f, t, api.SAMPLE_MAJOR)
        np.testing.assert_array_equal(cube, ref_cube)
        np.testing.assert_array_equal(w, ref_w)


def test_tensor_core_job_alone_equals_job_in_mix(ctx, tc_jobs):
    mix = run_batch(ctx, tc_jobs, [api.SAMPLE_MAJOR] * len(tc_jobs))
    for i in (1, 2, 3):
        alone = run_batch(ctx, [tc_jobs[i]], [api.SAMPLE_MAJOR])[0]
        np.testing.assert_array_equal(alone[0], mix[i][0])
        np.testing.assert_array_equal(alone[1], mix[i][1])


def test_batch_over_entry_budget_routes_jobs_to_single_path(ctx, jobs):
    """When a batch's entries exceed the context's entry budget, the jobs
    with the most entries run on the single-job path (in budget-sized
    passes) and the rest are batched: every cube still equals its single
    call."""
    ctx.set_entry_budget(2_000_000)  # bytes: 100,000 entries
    try:
        got = run_batch(ctx, jobs, [api.SAMPLE_MAJOR] * len(jobs))
    finally:
        ctx.set_entry_budget(4 << 30)
    for (job, f, t), (cube, w) in zip(jobs, got):
        ref_cube, ref_w = single(ctx, job, f, t, api.SAMPLE_MAJOR)
        np.testing.assert_array_equal(cube, ref_cube)
        np.testing.assert_array_equal(w, ref_w)
