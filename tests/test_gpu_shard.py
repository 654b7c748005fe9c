"""Dec-band sharding on one GPU: the bands of a job gridded one after
another from the sample ranges hcg_field_band_samples gives, assembled, equal
the whole map gridded at once (each band's pixels meet the same candidates in
the same order). On the FP32 engines that leaves the FP32 cube's rounding;
a band's FP16 tensor-core split takes its power-of-two channel scales from
the band's own spectra, so there the two results are each within the FP16
engine's 1e-5 of the FP64 cube, and within 2e-5 of each other. A map taller
than the data has bands that see no sample: NaN rows, weight 0, as the whole
map has them."""
import numpy as np
import pytest

from hcgrid_b200 import api, shard, synth

pytestmark = pytest.mark.gpu

TOL = {"single": 1e-6, api.ENGINE_FP32: 1e-6, api.ENGINE_TC_F16: 2e-5}  # of the plane's largest |value|


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def close(got, ref, w_got, w_ref, tol):
    nan = np.isnan(ref)
    assert np.array_equal(np.isnan(got), nan)
    ok = ~nan
    if ok.any():
        assert np.abs(got[ok] - ref[ok]).max() <= tol * np.abs(ref[ok]).max()
    np.testing.assert_allclose(w_got, w_ref, rtol=1e-6, atol=0)


def sharded(ctx, target, lon, lat, values, parts, weights=None, engine=api.ENGINE_AUTO):
    geo = ctx.field(lon, lat, weights)
    perm = geo.sorted()[1]
    bands = shard.plan(target.ny, parts)
    cube = np.empty((target.nx * target.ny, 1 if values.ndim == 1 else values.shape[1]), np.float32)
    w = np.empty(target.nx * target.ny, np.float32)
    sizes = []
    for y0, y1 in bands:
        s0, s1 = geo.band_samples(target, y0, y1)
        sizes.append(s1 - s0)
        c, ww = shard.grid_band(ctx, geo, target, lon, lat, values, y0, y1, weights=weights, engine=engine,
                                perm=perm)
        cube[y0 * target.nx:y1 * target.nx] = c
        w[y0 * target.nx:y1 * target.nx] = ww
    geo.close()
    return cube, w, sizes


@pytest.fixture(scope="module")
def job(ctx):
    j = synth.config2(n=60_000, nchan=70, nx=48, size_deg=1.0, build_values=True)
    t = ctx.target_from_header(j.header)
    yield j, t
    t.close()


@pytest.mark.parametrize("engine", ["single", api.ENGINE_FP32, api.ENGINE_TC_F16])
@pytest.mark.parametrize("kernel", ["gauss1d", "gauss2d_weighted"])
def test_bands_equal_whole_map(ctx, job, engine, kernel):
    j, t = job
    s = j.sigma_deg
    weights = None
    if kernel == "gauss1d":
        ctx.prepare_grid_kernel(api.GAUSS1D, np.array([s, 0.0, 0.0]), j.sphere_radius, j.hpx_max_res)
    else:
        ctx.prepare_grid_kernel(api.GAUSS2D, np.array([1.4 * s, 0.7 * s, 0.9]), j.sphere_radius, j.hpx_max_res)
        weights = np.random.default_rng(3).uniform(0.5, 2.0, j.n)
    values = np.ascontiguousarray(j.values[:, 0]) if engine == "single" else j.values
    eng = api.ENGINE_FP32 if engine == "single" else engine
    f = ctx.field(j.lon, j.lat, weights)
    f.set_spectra(values)
    if eng == api.ENGINE_TC_F16:
        f.split_spectra(eng)
    ref, wref = ctx.grid(f, t, engine=eng)
    f.close()
    cube, w, sizes = sharded(ctx, t, j.lon, j.lat, values, 3, weights=weights, engine=eng)
    assert 0 < max(sizes) < j.n  # each band took part of the samples
    close(cube, ref.reshape(cube.shape), w, wref, TOL[engine])


def test_bands_beyond_the_data_are_empty(ctx, job):
    """96 rows of 60" over data 1 deg high: the outer bands see no sample."""
    j, _ = job
    s = j.sigma_deg
    ctx.prepare_grid_kernel(api.GAUSS1D, np.array([s, 0.0, 0.0]), j.sphere_radius, j.hpx_max_res)
    t = ctx.target_from_header(synth.sin_header(48, 96, 180.0, 30.0, 1.0 / 48))
    values = np.ascontiguousarray(j.values[:, :8])
    f = ctx.field(j.lon, j.lat)
    f.set_spectra(values)
    ref, wref = ctx.grid(f, t)
    f.close()
    cube, w, sizes = sharded(ctx, t, j.lon, j.lat, values, 6)
    assert sizes[0] == 0 and sizes[-1] == 0 and min(sizes[1:-1]) > 0
    close(cube, ref, w, wref, TOL[api.ENGINE_FP32])
    assert np.isnan(cube[:16 * 48]).all() and (w[:16 * 48] == 0).all()
    t.close()
