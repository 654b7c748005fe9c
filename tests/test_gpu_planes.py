"""hcg_grid_planes: host channel planes in, host cube out, pipelined in
blocks of channels, against hcg_grid on the same spectra through the C ABI.

The FP32 engine sums every channel in the same order whatever the block, so
its planes cube equals hcg_grid's bit for bit. The tensor-core engines take a
pipeline shape per channel class, so a 64-channel block may run a different
shape than the whole field: those cubes agree to the FP32 accumulation's
rounding (1e-6 of each channel plane's largest value), and both stay within
the engines' 1e-5 of the FP32 engine. Weights are the same FP64 sums."""
import numpy as np
import pytest
import torch

from hcgrid_b200 import api, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def plane_errors(cube, ref):
    """max over channels of max|cube - ref| / max|ref|; cube, ref [npix, nchan]."""
    nan = np.isnan(ref)
    assert np.array_equal(np.isnan(cube), nan)
    worst = 0.0
    for c in range(ref.shape[1]):
        r = ref[~nan[:, c], c]
        if r.size:
            worst = max(worst, np.abs(cube[~nan[:, c], c].astype(np.float64) - r).max() / max(np.abs(r).max(), 1e-30))
    return worst


@pytest.fixture(scope="module")
def job(ctx):
    j = synth.config2(n=150_000, nchan=200, nx=96, size_deg=1.6, build_values=True)
    ctx.prepare_grid_kernel(api.GAUSS1D, np.array([j.sigma_deg, 0.0, 0.0]), j.sphere_radius, j.hpx_max_res)
    return j


@pytest.fixture(scope="module")
def whole(ctx, job):
    """hcg_grid on the whole field: FP32, and FP16 hi/lo ([npix, nchan] cubes)."""
    f = ctx.field(job.lon, job.lat)
    f.set_spectra(job.values)
    t = ctx.target_from_header(job.header)
    c32, w32 = ctx.grid(f, t, engine=api.ENGINE_FP32)
    f.split_spectra(api.ENGINE_TC_F16)
    c16, w16 = ctx.grid(f, t, engine=api.ENGINE_TC_F16)
    f.close()
    t.close()
    return c32, w32, c16, w16


def planes_of(job, nchan=None, pinned=False):
    v = job.values if nchan is None else job.values[:, :nchan]
    p = np.ascontiguousarray(v.T)  # [nchan][n], input sample order
    if pinned:
        t = torch.empty(p.shape, dtype=torch.float32, pin_memory=True)
        t.copy_(torch.from_numpy(p))
        return t
    return p


@pytest.mark.parametrize("block", [0, 64, 128])
def test_fp32_planes_equal_hcg_grid(ctx, job, whole, block):
    c32, w32, _, _ = whole
    g = ctx.field(job.lon, job.lat)
    t = ctx.target_from_header(job.header)
    try:
        cube, w = ctx.grid_planes(g, t, planes_of(job), engine=api.ENGINE_FP32, block=block)
    finally:
        g.close()
        t.close()
    np.testing.assert_array_equal(cube.T, c32)
    np.testing.assert_array_equal(w, w32)


@pytest.mark.parametrize("layout", [api.CHANNEL_MAJOR, api.SAMPLE_MAJOR])
@pytest.mark.parametrize("block", [0, 64])
def test_tc_planes_match_hcg_grid(ctx, job, whole, layout, block):
    """Pinned planes and cube (the overlapped copies), both cube layouts."""
    c32, w32, c16, w16 = whole
    planes = planes_of(job, pinned=True)
    P = c32.shape[0]
    shape = (job.nchan, P) if layout == api.CHANNEL_MAJOR else (P, job.nchan)
    cube = torch.empty(shape, dtype=torch.float32, pin_memory=True)
    w = torch.empty(P, dtype=torch.float32, pin_memory=True)
    g = ctx.field(job.lon, job.lat)
    t = ctx.target_from_header(job.header)
    try:
        ctx.grid_planes(g, t, planes, cube, w, layout=layout, engine=api.ENGINE_TC_F16, block=block)
    finally:
        g.close()
        t.close()
    c = cube.numpy()
    c = c.T if layout == api.CHANNEL_MAJOR else c
    np.testing.assert_allclose(w.numpy(), w16, rtol=1e-6)
    assert plane_errors(c, c16.astype(np.float64)) <= 1e-6
    assert plane_errors(c, c32.astype(np.float64)) <= 1e-5


def test_single_channel_last_block(ctx, job, whole):
    """129 channels in blocks of 64: the last block holds one channel, which
    takes the single-channel FP64 path (as hcg_grid does for a one-channel
    field), the others the tensor cores; all within 1e-5 of the FP32 engine."""
    c32, w32, _, _ = whole
    g = ctx.field(job.lon, job.lat)
    t = ctx.target_from_header(job.header)
    try:
        cube, w = ctx.grid_planes(g, t, planes_of(job, 129), engine=api.ENGINE_TC_F16, block=64)
    finally:
        g.close()
        t.close()
    assert plane_errors(cube.T, c32[:, :129].astype(np.float64)) <= 1e-5
    np.testing.assert_allclose(w, w32, rtol=1e-6)


def test_planes_refusals(ctx, job):
    g = ctx.field(job.lon, job.lat)
    t = ctx.target_from_header(job.header)
    try:
        with pytest.raises(RuntimeError, match="HCG_EINVAL"):
            ctx.grid_planes(g, t, planes_of(job, 64), block=100)  # not a multiple of 64
        with pytest.raises(RuntimeError, match="HCG_EINVAL"):
            ctx.grid_planes(g, t, planes_of(job, 64), layout=7)
        with pytest.raises(ValueError):
            ctx.grid_planes(g, t, torch.zeros((2, job.n), device="cuda"))
    finally:
        g.close()
        t.close()
